"""Flat-panel cone-beam projection and backprojection (drop-in for ``aprict.cb.flatpanel``).

Same names, arguments, accumulate semantics and exceptions as
src/aprict/cb/flatpanel.py:
  * ``ProjGeom`` (:269-768): per-view source, detector centre and pixel vectors,
    regularised to float32 on construction (:311-318, :612-622);
  * ``ProjectionSet`` (:771-882): a geometry plus a (..., M, nu, nv) float32
    (or float16 / float64, as the reference allows) device array (a torch
    tensor here, v fastest);
  * ``ConfigProject`` / ``ConfigBackproject`` (:885-994);
  * ``project`` (:997-1125) and ``backproject`` (:1128-1281), which ADD into
    their output.
The compute goes through the C ABI of libaprict_b200.so (sm_100a kernels);
there is no other implementation to fall back to.
"""

from __future__ import annotations

import dataclasses
import itertools
import json
import logging
import math
import pathlib

import numpy as np
import torch

from .. import _lib
from .. import _structs as S
from ..volume import FBVolume, Volume


def force_compile(*, log_stream: object | None = None) -> None:  # noqa: ARG001
    """Load the prebuilt kernel library (the reference JIT-compiles here, flatpanel.py:114-117)."""
    _lib.lib()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _device() -> torch.device:
    if not torch.cuda.is_available():
        msg = "aprict_b200 needs a CUDA device (B200, sm_100a); none is available"
        raise RuntimeError(msg)
    return torch.device("cuda", torch.cuda.current_device())


# --------------------------------------------------------------------------- geometry
def _assert_flatpanel_geometry_consistency(proj_specs: np.ndarray, data: torch.Tensor | None) -> tuple[int, ...]:
    """Validate a view array against a data buffer; return the expected data shape (flatpanel.py:235-266)."""
    if proj_specs.dtype != S.proj_spec:
        msg = "Invalid dtype for the input array. It should be an array of 'proj_spec' objects."
        raise ValueError(msg)
    if not np.all(proj_specs["type"] == 0):
        msg = "Only flat-panel detectors are currently supported. One or more of the provided proj_spec indicates a detector type other than flat panel."
        raise NotImplementedError(msg)
    nus = proj_specs["nu"].reshape(-1)
    nvs = proj_specs["nv"].reshape(-1)
    if nus.size and (not np.all(nus == nus[0]) or not np.all(nvs == nvs[0])):
        msg = "The input detector dimensions are inconsistent between projections. This is not currently implemented."
        raise NotImplementedError(msg)
    if proj_specs.ndim < 1:
        msg = "The input proj_specs array is not at least a 1D array. It should be at least a 1D array."
        raise ValueError(msg)
    det_shape = (int(nus[0]), int(nvs[0])) if nus.size else (0, 0)
    data_shape = tuple(proj_specs.shape) + det_shape
    if data is not None and tuple(data.shape) != data_shape:
        msg = f"Invalid shape for the output_array. The expected shape is {data_shape}, but the provided output_array has shape {tuple(data.shape)}."
        raise NotImplementedError(msg)
    return data_shape


@dataclasses.dataclass(kw_only=True, eq=False)
class ProjGeom:
    """Geometry of a set of flat-panel cone-beam projections."""

    source_pos: np.ndarray
    det_pos: np.ndarray
    det_uvec: np.ndarray
    det_vvec: np.ndarray
    nu: np.ndarray
    nv: np.ndarray

    def __init__(
        self,
        *,
        source_pos: np.ndarray,
        det_pos: np.ndarray,
        det_uvec: np.ndarray,
        det_vvec: np.ndarray,
        nu: int | np.integer | np.ndarray,
        nv: int | np.integer | np.ndarray,
        _skip_regularisation: bool = False,
    ) -> None:
        if _skip_regularisation:
            self.source_pos, self.det_pos, self.det_uvec, self.det_vvec = source_pos, det_pos, det_uvec, det_vvec
            self.nu, self.nv = nu, nv  # type: ignore[assignment]
            return
        vecs = [np.asarray(a) for a in (source_pos, det_pos, det_uvec, det_vvec)]
        ints = [np.asarray(a) for a in (nu, nv)]
        # Leading (projection-list) dims are padded with trailing 1s to a common
        # rank so that they broadcast (flatpanel.py:556-600), then cast to
        # float32/uint32 as the JSON round trip of the reference does (:612-622).
        pdim = max([a.ndim - 1 for a in vecs] + [a.ndim for a in ints])
        vecs = [a.reshape(a.shape[:-1] + (1,) * (pdim - (a.ndim - 1)) + (3,)).astype(np.float32) for a in vecs]
        ints = [a.reshape(a.shape + (1,) * (pdim - a.ndim)).astype(np.uint32) for a in ints]
        self.source_pos, self.det_pos, self.det_uvec, self.det_vvec = vecs
        self.nu, self.nv = ints

    # -------------------------------------------------------------- shape info
    @property
    def projs_list_shape(self) -> tuple[int, ...]:
        """Broadcast shape of the projection list (e.g. (M,))."""
        return tuple(
            np.broadcast_shapes(
                self.source_pos.shape[:-1],
                self.det_pos.shape[:-1],
                self.det_uvec.shape[:-1],
                self.det_vvec.shape[:-1],
                self.nu.shape,
                self.nv.shape,
            )
        )

    @property
    def num_projs(self) -> int:
        """The number of cone-beam projections."""
        return math.prod(self.projs_list_shape)

    def get_bbox(
        self, *, index_tuple: tuple[int, ...] | None = None
    ) -> tuple[tuple[float, float, float], tuple[float, float, float]]:
        """((minx,miny,minz),(maxx,maxy,maxz)) of the sources and detector corners (flatpanel.py:320-368)."""
        it = () if index_tuple is None else index_tuple
        axes = tuple(range(len(self.projs_list_shape) - len(it)))
        hu = self.det_uvec * self.nu[..., None] / 2
        hv = self.det_vvec * self.nv[..., None] / 2
        mins, maxs = [], []
        for pts in (self.source_pos, self.det_pos + hu + hv, self.det_pos + hu - hv, self.det_pos - hu + hv, self.det_pos - hu - hv):
            p = np.broadcast_to(pts, self.projs_list_shape + (3,))[it]
            mins.append(np.min(p, axis=axes))
            maxs.append(np.max(p, axis=axes))
        return tuple(np.min(np.stack(mins), axis=0).tolist()), tuple(np.max(np.stack(maxs), axis=0).tolist())  # type: ignore[return-value]

    # ----------------------------------------------------------- derived views
    def sliced(self, sl: slice | list[int]) -> ProjGeom:
        """A copy restricted to the projections selected by ``sl`` (flatpanel.py:387-425)."""
        if type(sl) not in (slice, list):
            msg = f"Invalid type for slice object {sl}"
            raise ValueError(msg)
        if len(self.projs_list_shape) != 1:
            msg = "Slicing has not been implemented for non-flat projection lists."
            raise NotImplementedError(msg)
        n = self.num_projs

        def f(a: np.ndarray) -> np.ndarray:
            if n == 1 or a.shape[0] != 1:
                return a[sl, ...].copy()
            return a.copy()

        return ProjGeom(
            source_pos=f(self.source_pos),
            det_pos=f(self.det_pos),
            det_uvec=f(self.det_uvec),
            det_vvec=f(self.det_vvec),
            nu=f(self.nu),
            nv=f(self.nv),
        )

    def flipped(self, *, flip_x: bool, flip_y: bool, flip_z: bool) -> ProjGeom:
        """Mirror the geometry along the chosen axes."""
        fl = np.array([-1 if flip_x else 1, -1 if flip_y else 1, -1 if flip_z else 1], dtype=np.float32)
        return ProjGeom(
            source_pos=self.source_pos * fl,
            det_pos=self.det_pos * fl,
            det_uvec=self.det_uvec * fl,
            det_vvec=self.det_vvec * fl,
            nu=self.nu,
            nv=self.nv,
        )

    def rotated(self, *, xy_rads: float) -> ProjGeom:
        """Rotate about the z axis."""
        c, s = np.cos(xy_rads), np.sin(xy_rads)
        rot = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], dtype=np.float32)
        r = lambda a: np.tensordot(a, rot, axes=(-1, -1))  # noqa: E731
        return ProjGeom(
            source_pos=r(self.source_pos),
            det_pos=r(self.det_pos),
            det_uvec=r(self.det_uvec),
            det_vvec=r(self.det_vvec),
            nu=self.nu,
            nv=self.nv,
        )

    def translated(self, *, x: float, y: float, z: float) -> ProjGeom:
        """Translate the sources and detectors."""
        t = np.array([x, y, z], dtype=np.float32)
        return ProjGeom(
            source_pos=self.source_pos + t,
            det_pos=self.det_pos + t,
            det_uvec=self.det_uvec,
            det_vvec=self.det_vvec,
            nu=self.nu,
            nv=self.nv,
        )

    def binned(self, *, n: int) -> ProjGeom:
        """The geometry of an n x n binned detector."""
        if not n > 0 or not (np.all(self.nu % n == 0) and np.all(self.nv % n == 0)):
            msg = "'n' should be a positive integer that divides all detector dimensions."
            raise ValueError(msg)
        return ProjGeom(
            source_pos=self.source_pos,
            det_pos=self.det_pos,
            det_uvec=self.det_uvec * n,
            det_vvec=self.det_vvec * n,
            nu=self.nu // n,
            nv=self.nv // n,
        )

    def __eq__(self, other: object) -> bool:
        if not isinstance(other, ProjGeom):
            return False
        return all(
            np.array_equal(getattr(self, k), getattr(other, k))
            for k in ("source_pos", "det_pos", "det_uvec", "det_vvec", "nu", "nv")
        )

    def __ne__(self, other: object) -> bool:
        return not self.__eq__(other)

    __hash__ = None  # type: ignore[assignment]

    # --------------------------------------------------------------- JSON I/O
    def json(self) -> dict:
        """A JSON-serialisable dict (same keys as the reference, flatpanel.py:534-610)."""
        return {
            "source_pos": self.source_pos.tolist(),
            "det_pos": self.det_pos.tolist(),
            "det_uvec": self.det_uvec.tolist(),
            "det_vvec": self.det_vvec.tolist(),
            "nu": self.nu.tolist(),
            "nv": self.nv.tolist(),
        }

    def json_str(self) -> str:
        """The JSON text of :meth:`json`."""
        return json.dumps(self.json(), indent=2)

    @staticmethod
    def _from_json_dict(d: dict) -> ProjGeom:
        return ProjGeom(
            source_pos=np.array(d["source_pos"], dtype=np.float32),
            det_pos=np.array(d["det_pos"], dtype=np.float32),
            det_uvec=np.array(d["det_uvec"], dtype=np.float32),
            det_vvec=np.array(d["det_vvec"], dtype=np.float32),
            nu=np.array(d["nu"], dtype=np.uint32),
            nv=np.array(d["nv"], dtype=np.uint32),
            _skip_regularisation=True,
        )

    @staticmethod
    def load(fpath: pathlib.Path | str) -> ProjGeom:
        """Load a geometry saved by :meth:`save` (or by the reference)."""
        fpath = pathlib.Path(fpath)
        if not fpath.exists():
            raise FileNotFoundError(fpath)
        with open(fpath, encoding="utf-8") as f:
            return ProjGeom._from_json_dict(json.load(f))

    def save(self, fpath: pathlib.Path | str, *, allow_overwrite: bool = False) -> None:
        """Save as JSON."""
        fpath = pathlib.Path(fpath)
        if not allow_overwrite and fpath.exists():
            raise FileExistsError(fpath)
        with open(fpath, mode="w+", encoding="utf-8") as f:
            f.write(self.json_str())

    def to_proj_spec_array(self) -> np.ndarray:
        """Pack into an array of proj_spec structs with shape ``projs_list_shape``."""
        shp = self.projs_list_shape
        out = np.zeros(shp, dtype=S.proj_spec)
        for name, arr in (
            ("source_pos", self.source_pos),
            ("det_pos", self.det_pos),
            ("det_u", self.det_uvec),
            ("det_v", self.det_vvec),
        ):
            b = np.broadcast_to(arr, shp + (3,))
            out[name]["x"], out[name]["y"], out[name]["z"] = b[..., 0], b[..., 1], b[..., 2]
        out["nu"] = np.broadcast_to(self.nu, shp)
        out["nv"] = np.broadcast_to(self.nv, shp)
        out["type"] = 0
        return out

    @classmethod
    def new_circular_scan(
        cls,
        *,
        num_source_points: int,
        R: float,  # noqa: N803
        L_minus_R: float,  # noqa: N803
        pix_widhei_at_isocenter: tuple[float, float],
        det_widhei: tuple[float, float] | None = None,
        num_pix_widhei: tuple[int, int] | None = None,
        theta_start: float = 0,
        theta_clockwise: bool = False,
        arc_length_rads: float = 2 * np.pi,
        isocenter: tuple[float, float, float] | np.ndarray = (0, 0, 0),
    ) -> ProjGeom:
        """A circular scan about the z axis (same construction as flatpanel.py:682-768)."""
        if (det_widhei is None) == (num_pix_widhei is None):
            msg = "Exactly one of 'det_widhei' and 'num_pix_widhei' must be specified."
            raise ValueError(msg)
        L = R + L_minus_R  # noqa: N806
        px, py = pix_widhei_at_isocenter
        if num_pix_widhei is None:
            dx, dy = det_widhei  # type: ignore[misc]
            num_pix_widhei = (math.ceil(dx / (px * L / R)), math.ceil(dy / (py * L / R)))
        pixel_wid, pixel_hei = (L / R) * px, (L / R) * py
        ts = np.linspace(
            theta_start,
            theta_start + arc_length_rads * (-1 if theta_clockwise else 1),
            endpoint=False,
            num=num_source_points,
            dtype=np.float64,
        )
        zs = np.zeros_like(ts)
        src = np.stack([R * np.cos(ts), R * np.sin(ts), zs], axis=-1)
        det = src * np.array([[1 - L / R, 1 - L / R, 1]])
        iso = np.asarray(isocenter, dtype=np.float64)[None, :]
        uvec = pixel_wid * np.stack([-np.sin(ts), np.cos(ts), 0 * ts], axis=-1)
        vvec = pixel_hei * np.array([[0, 0, -1]], dtype=np.float64)
        return cls(
            source_pos=src + iso,
            det_pos=det + iso,
            det_uvec=uvec,
            det_vvec=vvec,
            nu=num_pix_widhei[0],
            nv=num_pix_widhei[1],
        )


# --------------------------------------------------------------------------- data
# Projection data types of the reference's kernels (half, float, double; flatpanel.py:120-185).
# The kernels here compute in FP32: other types pass through FP32 working copies.
_PROJ_DTYPES = {np.dtype(np.float16): torch.float16, np.dtype(np.float32): torch.float32,
                np.dtype(np.float64): torch.float64}


def _np_dtype(t: torch.Tensor) -> np.dtype:
    return np.dtype(str(t.dtype).replace("torch.", ""))


class ProjectionSet:
    """A projection geometry with (optionally) its detector data on the GPU."""

    def __init__(self, pg: ProjGeom, *, data: np.ndarray | torch.Tensor | None) -> None:
        if data is not None:
            if isinstance(data, np.ndarray):
                if data.dtype not in _PROJ_DTYPES:
                    msg = f"Projection dtype {data.dtype} is not supported (float16, float32 or float64)."
                    raise NotImplementedError(msg)
                data = torch.from_numpy(np.ascontiguousarray(data)).to(_device())
            elif data.dtype not in _PROJ_DTYPES.values():
                msg = f"Projection dtype {data.dtype} is not supported (float16, float32 or float64)."
                raise NotImplementedError(msg)
            elif not data.is_cuda:
                data = data.to(_device())
        proj_specs = pg.to_proj_spec_array()
        _assert_flatpanel_geometry_consistency(proj_specs, data)
        self._proj_geom = pg
        self._proj_specs = proj_specs
        self._data = data
        self._specs_dev: torch.Tensor | None = None
        self._out_of_mem_counter: torch.Tensor | None = None

    def _with_data(self, data: torch.Tensor) -> ProjectionSet:
        """A ProjectionSet of this geometry over ``data`` (a device tensor of the same
        shape), sharing the packed views and their device copy (no re-packing or upload)."""
        _assert_flatpanel_geometry_consistency(self._proj_specs, data)
        out = ProjectionSet.__new__(ProjectionSet)
        out._proj_geom = self._proj_geom
        out._proj_specs = self._proj_specs
        out._data = data
        out._specs_dev = self.specs_device()
        out._out_of_mem_counter = None
        return out

    @property
    def proj_geom(self) -> ProjGeom:
        """The geometry."""
        return self._proj_geom

    @property
    def proj_specs(self) -> np.ndarray:
        """The packed views (proj_spec structs), shape ``projs_list_shape``."""
        return self._proj_specs

    @property
    def data(self) -> torch.Tensor | None:
        """The device data (not copied)."""
        return self._data

    def get_bbox(self, *, index_tuple: tuple[int, ...] | None = None) -> tuple:
        """Bounding box of the geometry (see ProjGeom.get_bbox)."""
        return self._proj_geom.get_bbox(index_tuple=index_tuple)

    @property
    def out_of_mem_counter(self) -> torch.Tensor:
        """Device uint32 word counting rays whose quadric interval list overflowed."""
        if self._out_of_mem_counter is None:
            self._out_of_mem_counter = torch.zeros(1, dtype=torch.int32, device=_device())
        return self._out_of_mem_counter

    @property
    def out_of_mem_counter_cp(self) -> torch.Tensor:
        """The overflow counter under the reference's name (a (1,) device array; a torch tensor here)."""
        return self.out_of_mem_counter

    @property
    def out_of_mem_count(self) -> int:
        """Number of overflowed rays (flatpanel.py:817-820)."""
        return int(self.out_of_mem_counter.item())

    def specs_device(self) -> torch.Tensor:
        """The packed views on the device (uint8 bytes, flattened), cached."""
        if self._specs_dev is None:
            raw = np.ascontiguousarray(self._proj_specs.reshape(-1)).view(np.uint8)
            _device()
            self._specs_dev = _lib.upload(raw)
        return self._specs_dev

    def create_buffer(self, *, dtype: type | np.dtype = np.float32, existing_ok: bool = False) -> None:
        """Allocate a zero-filled data buffer."""
        if self._data is not None:
            if existing_ok:
                return
            msg = "Data buffer already exists. Pass 'existing_ok=True' to allow this to occur without raising an exception."
            raise RuntimeError(msg)
        if np.dtype(dtype) not in _PROJ_DTYPES:
            msg = f"Projection dtype {np.dtype(dtype)} is not supported (float16, float32 or float64)."
            raise NotImplementedError(msg)
        shape = _assert_flatpanel_geometry_consistency(self._proj_specs, None)
        self._data = torch.zeros(shape, dtype=_PROJ_DTYPES[np.dtype(dtype)], device=_device())

    def zeroed_copy(self, dtype: type | np.dtype | None = None) -> ProjectionSet:
        """A copy with a zero-filled buffer."""
        if self._data is None and dtype is None:
            msg = "Cannot create a zeroed copy without an explicit 'dtype' argument, because the object you are trying to copy does not yet have a determined dtype."
            raise ValueError(msg)
        ps = ProjectionSet(self._proj_geom, data=None)
        ps._specs_dev = self._specs_dev
        ps.create_buffer(dtype=_np_dtype(self._data) if dtype is None else dtype)
        return ps


# --------------------------------------------------------------------------- configs
class ConfigProject:
    """Settings for :func:`project` (flatpanel.py:885-926)."""

    def __init__(
        self,
        *,
        shrink_volume_factor: float | None = None,
        multiply_before_adding: float | None = None,
        ssu: int | None = None,
        ssv: int | None = None,
        overlap_addition: bool = False,
        additive_line_integral: bool = False,
    ) -> None:
        # `x or 1` as in the reference: None and 0 both mean 1.
        svf = shrink_volume_factor or 1
        mba = multiply_before_adding or 1
        ssu = ssu or 1
        ssv = ssv or 1
        self._contents = np.array((np.float32(svf), np.float32(mba), np.uint32(ssu), np.uint32(ssv)), dtype=S.project_config)
        # FORBILD path: later shapes take priority unless overlap_addition
        # (flatpanel.py:917-926; the reference hard-codes False).
        self._overlap_addition = bool(overlap_addition)
        # additive mode in length units (sum rho * chord) instead of the
        # reference's parametric sum (sum rho * dt)
        self.additive_line_integral = bool(additive_line_integral)

    @property
    def contents(self) -> np.ndarray:
        """The packed aprict_project_config."""
        return self._contents.copy()

    @property
    def overlap_addition(self) -> bool:
        """Whether overlapping FORBILD shapes add instead of the last one winning."""
        return self._overlap_addition


class ConfigBackproject:
    """Settings for :func:`backproject` (flatpanel.py:929-994); defaults give the exact adjoint."""

    def __init__(
        self,
        *,
        fast_approx: bool = False,
        cyl_mask_rad: float | None = None,
        backproject_1s: bool = False,
        apply_summand_multiplier: bool = False,
        soften_det_edges_proportion: float | None = None,
        Z_on_L_factor_power: int = 0,  # noqa: N803
        Z_on_val_factor_power: int = 0,  # noqa: N803
        Z_on_val_factor_val: float = 1,  # noqa: N803
        approx_mode_direct_raycast: bool = False,
        approx_mode_bilinear_interpolate: bool = False,
        backproj_weighting_preset: int = 0,
        ssx: int = 1,
        ssy: int = 1,
        ssz: int = 1,
        soft_vartheta_v: float | None = None,
        soft_vartheta_v_softspan: float | None = None,
        soft_vartheta_h: float | None = None,
        soft_vartheta_h_softspan: float | None = None,
    ) -> None:
        r = cyl_mask_rad or 0
        sep = soften_det_edges_proportion or 0
        self._contents = np.array(
            (
                np.uint32(not fast_approx),
                np.uint32(bool(backproject_1s)),
                np.uint32(bool(r)),
                np.float32(r),
                np.uint32(bool(apply_summand_multiplier)),
                np.float32(sep),
                np.int32(Z_on_L_factor_power),
                np.int32(Z_on_val_factor_power),
                np.float32(Z_on_val_factor_val),
                np.uint32(bool(approx_mode_direct_raycast)),
                np.uint32(bool(approx_mode_bilinear_interpolate)),
                np.uint32(backproj_weighting_preset),
                np.uint32(ssx),
                np.uint32(ssy),
                np.uint32(ssz),
                np.float32(soft_vartheta_v or 0),
                np.float32(soft_vartheta_v_softspan or 0),
                np.float32(soft_vartheta_h or 0),
                np.float32(soft_vartheta_h_softspan or 0),
            ),
            dtype=S.backproject_config,
        )

    @property
    def contents(self) -> np.ndarray:
        """The packed aprict_backproject_config."""
        return self._contents.copy()


# --------------------------------------------------------------------------- operators
def _leading_slices(projs: ProjectionSet) -> list[tuple[tuple[int, ...], int]]:
    """(index tuple, flat index of its first view) for every leading index tuple."""
    lead = projs.proj_specs.shape[:-1]
    m = projs.proj_specs.shape[-1]
    return [(it, int(np.ravel_multi_index(it, lead)) * m if lead else 0) for it in itertools.product(*map(range, lead))]


def _view_args(projs: ProjectionSet, it: tuple[int, ...], first: int,
               data: torch.Tensor | None = None) -> tuple[int, np.ndarray, int]:
    data = projs.data if data is None else data
    assert data is not None
    sub = data[it] if it else data
    m, nu, nv = sub.shape[-3:]
    pd = _lib.proj_desc((m, nu, nv), tuple(sub.stride()[-3:]))
    specs = projs.specs_device().data_ptr() + first * S.proj_spec.itemsize
    return specs, pd, sub.data_ptr()


def _f32_twin(projs: ProjectionSet) -> ProjectionSet:
    """``projs`` itself when its data is float32, else a zero-filled float32
    twin with the same geometry (and overflow counter) for the kernels to add
    into; :func:`_fold_twin` adds it back."""
    assert projs.data is not None
    if projs.data.dtype == torch.float32:
        return projs
    tw = ProjectionSet(projs.proj_geom, data=torch.zeros(projs.data.shape, dtype=torch.float32, device=projs.data.device))
    tw._specs_dev = projs._specs_dev  # noqa: SLF001
    tw._out_of_mem_counter = projs.out_of_mem_counter  # noqa: SLF001
    return tw


def _fold_twin(projs: ProjectionSet, tw: ProjectionSet) -> None:
    """projs.data += tw.data in projs' own dtype (exact for float64, one rounding for float16)."""
    if tw is not projs:
        assert projs.data is not None and tw.data is not None
        projs.data.add_(tw.data.to(projs.data.dtype) if projs.data.dtype == torch.float64 else tw.data)


def _f32_data(t: torch.Tensor) -> torch.Tensor:
    """A float32 tensor with t's values and strides: t itself, or a converted copy."""
    return t if t.dtype == torch.float32 else t.float()


def _check_volume_device(volume: Volume) -> None:
    if not volume.data.is_cuda:
        msg = "Volume data must live on the GPU."
        raise ValueError(msg)


def project(
    config: ConfigProject,
    volume: Volume | FBVolume,
    projs: ProjectionSet,
    block: bool = False,
) -> ProjectionSet:
    """Add the projection of ``volume`` into ``projs`` (flatpanel.py:997-1125)."""
    projs.create_buffer(dtype=np.float32, existing_ok=True)
    work = _f32_twin(projs)  # float16 / float64 data: project into float32, then add
    if type(volume) is FBVolume:
        from . import forbild  # noqa: PLC0415

        forbild.project_shapes(config, volume, work)
    elif type(volume) is Volume:
        _check_volume_device(volume)
        cfg = config.contents
        vd = volume._desc()  # noqa: SLF001
        v32 = volume._f32()  # noqa: SLF001
        for it, first in _leading_slices(work):
            specs, pd, dptr = _view_args(work, it, first)
            _lib.check(
                _lib.lib().aprict_b200_project_siddon(
                    specs, _lib.ptr(pd), dptr, None, _lib.ptr(vd), v32.data_ptr(), _lib.ptr(cfg), None, _stream()
                ),
                "project",
            )
    else:
        msg = f"Unknown volume type: {type(volume)}"
        raise RuntimeError(msg)
    _fold_twin(projs, work)
    if block:
        torch.cuda.current_stream().synchronize()
    return projs


def project_residual(config: ConfigProject, volume: Volume, projs: ProjectionSet, base: torch.Tensor) -> ProjectionSet:
    """``projs.data = base + mba * A volume`` in one pass (no separate copy of ``base``).

    With ``multiply_before_adding=-1`` this is the residual b - A x that the
    reference forms as copyto + project (sirt_vram.py:133-140).
    """
    projs.create_buffer(dtype=np.float32, existing_ok=True)
    assert projs.data is not None
    if tuple(base.shape) != tuple(projs.data.shape) or base.stride() != projs.data.stride():
        msg = "base must have the shape and strides of the projection data"
        raise ValueError(msg)
    cfg = config.contents
    vd = volume._desc()  # noqa: SLF001
    v32, b32 = volume._f32(), _f32_data(base)  # noqa: SLF001
    out = _f32_data(projs.data)
    for it, first in _leading_slices(projs):
        specs, pd, dptr = _view_args(projs, it, first, data=out)
        bsub = b32[it] if it else b32
        _lib.check(
            _lib.lib().aprict_b200_project_siddon(
                specs, _lib.ptr(pd), dptr, bsub.data_ptr(), _lib.ptr(vd), v32.data_ptr(), _lib.ptr(cfg), None, _stream()
            ),
            "project_residual",
        )
    if out is not projs.data:
        projs.data.copy_(out)
    return projs


def backproject(
    config: ConfigBackproject,
    volume: Volume,
    projs: ProjectionSet,
    block: bool = False,
    summand_multiplier: Volume | None = None,
    logger: logging.Logger | None = None,  # noqa: ARG001
    enable_pbar: bool = False,  # noqa: ARG001
    secondary_volume: Volume | None = None,
) -> Volume:
    """Add the backprojection of ``projs`` into ``volume`` (flatpanel.py:1128-1281)."""
    if projs.data is None:
        msg = "You must provide projection data to this method."
        raise ValueError(msg)
    if summand_multiplier is not None:
        if summand_multiplier.shape != volume.shape:
            msg = f"Shape mismatch between volume and multiplier. Volume shape: {volume.shape}. Multiplier shape: {summand_multiplier.shape}"
            raise ValueError(msg)
        if summand_multiplier.dtype != volume.dtype or summand_multiplier.order != volume.order:
            msg = "dtype/order mismatch between summand multiplier and the volume is not implemented."
            raise NotImplementedError(msg)
    cfg = config.contents
    if bool(cfg["apply_summand_multiplier"]) != (summand_multiplier is not None):
        msg = "To prevent unintended behaviour, the config 'apply_summand_multiplier' must be true if and only if a summand_multiplier is included."
        raise ValueError(msg)
    preset = int(cfg["weighting_preset"])
    if preset > 7:
        msg = f"Backprojection weighting preset {preset} is not implemented."
        raise NotImplementedError(msg)
    _check_volume_device(volume)
    vd = volume._desc()  # noqa: SLF001
    # FP32 working copies of float16 volumes / non-FP32 projections (the kernels compute in FP32)
    v32 = volume._f32()  # noqa: SLF001
    m32 = summand_multiplier._f32() if summand_multiplier is not None else None  # noqa: SLF001
    mptr = m32.data_ptr() if m32 is not None else None
    p32 = _f32_data(projs.data)
    if preset == 7:
        # the GBC kernel, with the weight sums in the secondary volume (flatpanel.py:216-232)
        if secondary_volume is None:
            msg = "Weighting preset 7 (GBC) needs a secondary_volume to receive the sums of the weights."
            raise ValueError(msg)
        if secondary_volume.shape != volume.shape or secondary_volume.order != volume.order:
            msg = "The secondary volume must have the volume's shape and memory order."
            raise ValueError(msg)
        _check_volume_device(secondary_volume)
        s32 = secondary_volume._f32()  # noqa: SLF001
        for it, first in _leading_slices(projs):
            specs, pd, dptr = _view_args(projs, it, first, data=p32)
            _lib.check(
                _lib.lib().aprict_b200_backproject_gbc(
                    specs, _lib.ptr(pd), dptr, _lib.ptr(vd), v32.data_ptr(), s32.data_ptr(),
                    mptr, _lib.ptr(cfg), None, _stream(),
                ),
                "backproject_gbc",
            )
        volume._commit(v32)  # noqa: SLF001
        secondary_volume._commit(s32)  # noqa: SLF001
        if block:
            torch.cuda.current_stream().synchronize()
        return volume
    for it, first in _leading_slices(projs):
        specs, pd, dptr = _view_args(projs, it, first, data=p32)
        _lib.check(
            _lib.lib().aprict_b200_backproject(
                specs, _lib.ptr(pd), dptr, _lib.ptr(vd), v32.data_ptr(), mptr, _lib.ptr(cfg), None, _stream()
            ),
            "backproject",
        )
    volume._commit(v32)  # noqa: SLF001
    if block:
        torch.cuda.current_stream().synchronize()
    return volume


def backproject_adjoint(
    config: ConfigProject, volume: Volume, projs: ProjectionSet, block: bool = False
) -> Volume:
    """``volume += A^T projs`` for the Siddon operator of ``project(config, ...)``.

    Ray-driven scatter with the forward projector's own intersection lengths,
    so <A x, y> == <x, A^T y> up to float summation order.
    """
    if projs.data is None:
        msg = "You must provide projection data to this method."
        raise ValueError(msg)
    _check_volume_device(volume)
    cfg = config.contents
    vd = volume._desc()  # noqa: SLF001
    v32, p32 = volume._f32(), _f32_data(projs.data)  # noqa: SLF001
    for it, first in _leading_slices(projs):
        specs, pd, dptr = _view_args(projs, it, first, data=p32)
        _lib.check(
            _lib.lib().aprict_b200_backproject_scatter(
                specs, _lib.ptr(pd), dptr, _lib.ptr(vd), v32.data_ptr(), _lib.ptr(cfg), None, _stream()
            ),
            "backproject_adjoint",
        )
    volume._commit(v32)  # noqa: SLF001
    if block:
        torch.cuda.current_stream().synchronize()
    return volume


__all__ = [
    "ConfigBackproject",
    "ConfigProject",
    "ProjGeom",
    "ProjectionSet",
    "backproject",
    "backproject_adjoint",
    "force_compile",
    "project",
    "project_residual",
]
