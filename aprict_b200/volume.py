"""Voxel volumes (``Volume``) and analytic FORBILD phantoms (``FBVolume``).

Mirrors ``aprict.volume`` (src/aprict/volume/volume.py:51-495). The reference
stores a ``Volume`` in a CUDA array behind a surface object; users never touch
the texture (src/aprict/volume/volume.py:18-20), so here the storage is a
linear device buffer (a torch tensor with C- or F-order strides) that the
kernels index directly: float32, or float16 as the reference also allows
(:44-45). The kernels compute in FP32; a float16 volume is read through an
FP32 working copy and written back rounded (element-wise operations, the
projector and the backprojector alike). Voxel centres follow the reference convention:
``pos_c + voxwid * (i - (n-1)/2)`` (volume.py:133-145).
"""

from __future__ import annotations

import os

import pathlib
import typing

import numpy as np
import torch

from . import _lib

_SUPPORTED_DTYPES = (np.dtype(np.float32), np.dtype(np.float16))
_TORCH_DTYPES = {np.dtype(np.float32): torch.float32, np.dtype(np.float16): torch.float16}


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _device() -> torch.device:
    if not torch.cuda.is_available():
        msg = "aprict_b200 needs a CUDA device (B200, sm_100a); none is available"
        raise RuntimeError(msg)
    return torch.device("cuda", torch.cuda.current_device())


def _to_cupy(t: torch.Tensor) -> object:
    try:
        import cupy as cp  # noqa: PLC0415
    except ImportError as e:
        msg = "this method returns CuPy arrays and needs CuPy; the torch-returning method beside it does not"
        raise ImportError(msg) from e
    return cp.from_dlpack(t)


def _from_cupy(a: object) -> torch.Tensor:
    return torch.from_dlpack(a)


def _empty(shape: tuple[int, int, int], order: str, dtype: torch.dtype = torch.float32) -> torch.Tensor:
    X, Y, Z = shape
    strides = (Y * Z, Z, 1) if order == "C" else (1, X, X * Y)
    return torch.empty_strided(shape, strides, dtype=dtype, device=_device())


class Volume:
    """A rectangular prism of voxels, stored on the GPU."""

    _shape: tuple[int, int, int]
    _dtype: np.dtype
    _order: typing.Literal["C", "F"]
    _data: torch.Tensor
    _pos_c: np.ndarray
    _voxwid: float

    def __init__(
        self,
        arr: np.ndarray | torch.Tensor,
        *,
        voxwid: float,
        pos_c: np.ndarray | tuple[float, float, float] = (0.0, 0.0, 0.0),
        initialize_texture: bool = True,
        order: typing.Literal["C", "F"] = "C",
    ) -> None:
        if order not in ("C", "F"):
            msg = f"order must be 'C' or 'F', not {order!r}"
            raise ValueError(msg)
        if tuple(arr.shape).__len__() != 3:
            msg = "Volume arrays must be 3-dimensional (X, Y, Z)."
            raise ValueError(msg)
        dt = np.dtype(str(arr.dtype).replace("torch.", ""))
        if dt not in _SUPPORTED_DTYPES:
            msg = f"Volume dtype {dt} is not supported (float32 or float16)."
            raise NotImplementedError(msg)
        self._dtype = dt
        self._shape = tuple(int(s) for s in arr.shape)  # type: ignore[assignment]
        self._order = order
        self._voxwid = float(voxwid)
        self._pos_c = np.array(pos_c, dtype=np.float32).reshape(3)
        if initialize_texture:
            self._data = _empty(self._shape, order, _TORCH_DTYPES[dt])
            self.copy_from(arr)

    # ------------------------------------------------------------------ props
    @property
    def voxwid(self) -> float:
        """The width of each voxel."""
        return self._voxwid

    @property
    def shape(self) -> tuple[int, int, int]:
        """The shape (X, Y, Z) of the volume."""
        return self._shape

    @property
    def dtype(self) -> np.dtype:
        """The dtype of the volume."""
        return self._dtype

    @property
    def order(self) -> str:
        """Memory order of the device buffer: 'C' (z fastest) or 'F' (x fastest)."""
        return self._order

    @property
    def data(self) -> torch.Tensor:
        """The device tensor (shape (X,Y,Z), strides per ``order``); shared, not copied."""
        return self._data

    @property
    def pos_c(self) -> np.ndarray:
        """Position of the centre of the volume."""
        return self._pos_c.copy()

    @property
    def corner(self) -> np.ndarray:
        """World position of the outer corner of voxel (0,0,0) (flatpanel.py:1030-1036)."""
        return self._pos_c - np.float32(self._voxwid) * np.array(self._shape, dtype=np.float32) / 2

    @property
    def norm(self) -> float:
        """The l2 norm of the volume (double accumulation)."""
        return float(np.sqrt(self.inner_product(self)))

    @property
    def xs_ys_zs(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Voxel-centre coordinates along each axis."""
        out = []
        for a in range(3):
            n = self._shape[a]
            out.append(self._pos_c[a] + self._voxwid * (np.arange(n, dtype=np.float32) - (n - 1) / 2))
        return tuple(out)  # type: ignore[return-value]

    @property
    def minxyz_maxxyz(self) -> tuple[tuple[float, float, float], tuple[float, float, float]]:
        """Boundary tuple ((minx,miny,minz),(maxx,maxy,maxz))."""
        xs, ys, zs = self.xs_ys_zs
        h = self._voxwid / 2
        return (
            (float(xs.min() - h), float(ys.min() - h), float(zs.min() - h)),
            (float(xs.max() + h), float(ys.max() + h), float(zs.max() + h)),
        )

    # ------------------------------------------------------------ descriptors
    def _desc(self) -> np.ndarray:
        return _lib.vol_desc(self._shape, self._order, self._voxwid, self.corner)

    def _f32(self) -> torch.Tensor:
        """The data as float32 with the same strides: the tensor itself, or a copy of a float16 volume."""
        return self._data if self._data.dtype == torch.float32 else self._data.float()

    def _commit(self, t: torch.Tensor) -> None:
        """Store a float32 working copy from :meth:`_f32` back (a no-op when it is the data itself)."""
        if t is not self._data:
            self._data.copy_(t)

    @property
    def _numel(self) -> int:
        return int(np.prod(self._shape))

    # --------------------------------------------------------------- elementwise
    def fill(self, value: float) -> None:
        """Fill the volume with a constant value."""
        w = self._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_fill(w.data_ptr(), self._numel, float(value), _stream()),
            "Volume.fill",
        )
        self._commit(w)

    def multiply(self, f: float) -> None:
        """Multiply the volume in place by a value."""
        w = self._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_scale(w.data_ptr(), self._numel, float(f), _stream()),
            "Volume.multiply",
        )
        self._commit(w)

    def invert(self, *, ignore_zeros: bool = False, softmax_epsilon: float | None = None) -> None:
        """v <- 1/(v + eps exp(-v/eps)) (texture_tools.operations.invert, operations.py:347-374)."""
        w = self._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_invert(
                w.data_ptr(), self._numel, int(bool(ignore_zeros)), float(softmax_epsilon or 0), _stream()
            ),
            "Volume.invert",
        )
        self._commit(w)

    def multiply_volume(self, other: Volume) -> None:
        """Element-wise product with another volume of the same shape and order."""
        self._check_same(other)
        w, o = self._f32(), other._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_mul(w.data_ptr(), w.data_ptr(), o.data_ptr(), self._numel, _stream()),
            "Volume.multiply_volume",
        )
        self._commit(w)

    def divide(self, other: Volume) -> None:
        """Element-wise division by another volume (divide_textures)."""
        self.divide_softzero(other, eps=0.0)

    def divide_softzero(self, other: Volume, eps: float) -> None:
        """self <- self / (other + eps exp(-other / eps)) (volume.py:196-200,
        divide_surfaces_softzero); eps <= 0 divides plainly."""
        self._check_same(other)
        w, o = self._f32(), other._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_div_softzero(
                w.data_ptr(), w.data_ptr(), o.data_ptr(), self._numel, float(eps), _stream()
            ),
            "Volume.divide_softzero",
        )
        self._commit(w)

    def multiply_by_xygrid(self, xygrid: np.ndarray | torch.Tensor) -> None:
        """Multiply in place by an (nx, ny) grid broadcast over z (volume.py:170-190)."""
        g = torch.as_tensor(xygrid, dtype=torch.float32).to(self._data.device).contiguous()
        if tuple(g.shape) != tuple(self._shape[:2]):
            msg = "Input array should be 2-dimensional and match the shape[:2] of this volume."
            raise ValueError(msg)
        vd = self._desc()
        w = self._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_mul_xygrid(w.data_ptr(), _lib.ptr(vd), g.data_ptr(), _stream()),
            "Volume.multiply_by_xygrid",
        )
        self._commit(w)

    def add_scaled(self, other: Volume, alpha: float) -> None:
        """self += alpha * other."""
        self._check_same(other)
        w, o = self._f32(), other._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_axpy(w.data_ptr(), w.data_ptr(), float(alpha), o.data_ptr(), self._numel, _stream()),
            "Volume.add_scaled",
        )
        self._commit(w)

    def inner_product(self, other: Volume) -> float:
        """<self, other> accumulated in double on the device."""
        self._check_same(other)
        out = torch.zeros((), dtype=torch.float64, device=self._data.device)
        a, b = self._f32(), other._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_dot(a.data_ptr(), b.data_ptr(), self._numel, out.data_ptr(), _stream()),
            "Volume.inner_product",
        )
        return float(out.item())

    def soften_to_xy_cylinder(self, relrad_start: float) -> None:
        """Soft-mask to a cylinder coaxial with the volume's z axis (operations.py:377-401)."""
        if not 0 <= relrad_start <= 1:
            msg = "The input 'relrad_start' should be between 0 and 1."
            raise ValueError(msg)
        d = self._desc()
        w = self._f32()
        _lib.check(
            _lib.lib().aprict_b200_vol_softmask_cylinder(w.data_ptr(), _lib.ptr(d), float(relrad_start), _stream()),
            "Volume.soften_to_xy_cylinder",
        )
        self._commit(w)

    def _check_same(self, other: Volume) -> None:
        if other.shape != self.shape:
            msg = f"Shape mismatch: {self.shape} vs {other.shape}"
            raise ValueError(msg)
        if other.order != self.order:
            msg = "Volumes of different memory order are not supported in element-wise operations."
            raise NotImplementedError(msg)

    # ----------------------------------------------------------------- copies
    def copy_from(self, arr: np.ndarray | torch.Tensor, block: bool = True) -> None:
        """Copy a host/device array of shape (X,Y,Z) into this volume."""
        if tuple(arr.shape) != self._shape:
            msg = f"Shape mismatch: expected {self._shape}, got {tuple(arr.shape)}"
            raise ValueError(msg)
        src = arr if isinstance(arr, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32))
        self._data.copy_(src.to(self._data.dtype), non_blocking=not block)
        if block:
            torch.cuda.current_stream().synchronize()

    def copy_to(self, arr: np.ndarray | torch.Tensor, block: bool = True) -> None:
        """Copy this volume into a host/device array of shape (X,Y,Z)."""
        if isinstance(arr, torch.Tensor):
            arr.copy_(self._data, non_blocking=not block)
        else:
            arr[...] = self._data.cpu().numpy()
        if block:
            torch.cuda.current_stream().synchronize()

    def as_numpy(self, out: np.ndarray | None = None, allow_indirect_copy: bool = False) -> np.ndarray:  # noqa: ARG002
        """Copy this volume into a numpy array."""
        host = self._data.cpu().numpy()
        if out is None:
            return np.array(host, order=self._order)
        out[...] = host
        return out

    def as_torch(self) -> torch.Tensor:
        """A device copy of the volume as a torch tensor."""
        return self._data.clone()

    def as_cupy(self, out: object | None = None) -> object:  # noqa: ARG002
        """A CuPy view of the data (requires CuPy; zero-copy through DLPack)."""
        try:
            import cupy as cp  # noqa: PLC0415
        except ImportError as e:
            msg = "as_cupy needs CuPy; use as_torch() or .data instead"
            raise ImportError(msg) from e
        return cp.from_dlpack(self._data)

    def slice_axis(self, axis: int, sl: slice, *, out: torch.Tensor | None = None) -> torch.Tensor:
        """A C-contiguous device copy of the voxels ``sl`` along ``axis`` (3-D, this volume's dtype;
        slice_nth_axis_to_3d_cupy_array, operations.py:404-488)."""
        if sl.step not in (None, 1):
            msg = "Cannot use this method with a step size other than 1."
            raise NotImplementedError(msg)
        if axis not in (0, 1, 2):
            msg = "Invalid choice of axis. Choose 0, 1 or 2."
            raise ValueError(msg)
        start = 0 if sl.start is None else sl.start
        stop = self._shape[axis] if sl.stop is None else min(sl.stop, self._shape[axis])
        if stop - start <= 0:
            msg = f"Slice is empty. Provided slice: {sl}. Array shape: {self._shape}"
            raise ValueError(msg)
        idx = [slice(None)] * 3
        idx[axis] = slice(start, stop)
        src = self._data[tuple(idx)]
        if out is None:
            return src.contiguous() if not src.is_contiguous() else src.clone()
        if tuple(out.shape) != tuple(src.shape) or out.dtype != src.dtype or not out.is_contiguous():
            msg = f"Output must be a C-contiguous {src.dtype} tensor of shape {tuple(src.shape)}."
            raise ValueError(msg)
        out.copy_(src)
        return out

    def sum_axis(self, axis: int, *, out: torch.Tensor | None = None) -> torch.Tensor:
        """The volume summed along ``axis`` into a 2-D device tensor of this volume's dtype
        (accumulated in FP64; sum_along_nth_axis_to_2d_cupy_array, operations.py:491-560)."""
        if axis not in (0, 1, 2):
            msg = "Invalid choice of axis. Choose 0, 1 or 2."
            raise ValueError(msg)
        s = self._data.sum(dim=axis, dtype=torch.float64).to(self._data.dtype)
        if out is None:
            return s.contiguous()
        if tuple(out.shape) != tuple(s.shape) or out.dtype != s.dtype:
            msg = f"Output must be a {s.dtype} tensor of shape {tuple(s.shape)}."
            raise ValueError(msg)
        out.copy_(s)
        return out

    def as_cupy_slice(self, axis: int, sl: slice, *, out: object | None = None) -> object:
        """:meth:`slice_axis` as a CuPy array (requires CuPy; zero-copy through DLPack)."""
        return _to_cupy(self.slice_axis(axis, sl, out=None if out is None else _from_cupy(out)))

    def sum_to_cupy_array(self, axis: int, *, out: object | None = None) -> object:
        """:meth:`sum_axis` as a CuPy array (requires CuPy; zero-copy through DLPack)."""
        return _to_cupy(self.sum_axis(axis, out=None if out is None else _from_cupy(out)))

    def save(self, path: pathlib.Path | str) -> None:
        """Save the volume to a .npy file."""
        np.save(path, self.as_numpy())

    # ------------------------------------------------------------ constructors
    @classmethod
    def zeros(
        cls,
        shape: tuple[int, int, int],
        *,
        voxwid: float,
        dtype: type | np.dtype = np.float32,
        pos_c: np.ndarray | tuple[float, float, float] = (0.0, 0.0, 0.0),
        initialize_texture: bool = True,
        order: typing.Literal["C", "F"] = "C",
    ) -> Volume:
        """A new zero-filled volume (``initialize_texture=False`` allocates nothing)."""
        if type(shape) is not tuple or len(shape) != 3:
            msg = "Invalid shape provided. It should be a tuple of three positive integers."
            raise ValueError(msg)
        if np.dtype(dtype) not in _SUPPORTED_DTYPES:
            msg = f"Volume dtype {np.dtype(dtype)} is not supported (float32 or float16)."
            raise NotImplementedError(msg)
        self = cls.__new__(cls)
        self._shape = tuple(int(s) for s in shape)  # type: ignore[assignment]
        self._dtype = np.dtype(dtype)
        self._order = order
        self._voxwid = float(voxwid)
        self._pos_c = np.array(pos_c, dtype=np.float32).reshape(3)
        if initialize_texture:
            self._data = _empty(self._shape, order, _TORCH_DTYPES[self._dtype])
            self._data.zero_()
        return self

    @classmethod
    def from_tensor(
        cls,
        t: torch.Tensor,
        *,
        voxwid: float,
        pos_c: np.ndarray | tuple[float, float, float] = (0.0, 0.0, 0.0),
    ) -> Volume:
        """Wrap a float32 or float16 CUDA tensor of shape (X,Y,Z) without copying (C- or F-contiguous)."""
        if t.dim() != 3 or t.dtype not in (torch.float32, torch.float16) or not t.is_cuda:
            msg = "from_tensor needs a 3-D float32 or float16 CUDA tensor"
            raise ValueError(msg)
        X, Y, Z = t.shape  # noqa: N806
        if t.stride() == (Y * Z, Z, 1):
            order = "C"
        elif t.stride() == (1, X, X * Y):
            order = "F"
        else:
            msg = "from_tensor needs a C- or F-contiguous tensor"
            raise ValueError(msg)
        self = cls.__new__(cls)
        self._shape = (int(X), int(Y), int(Z))
        self._dtype = np.dtype(np.float32 if t.dtype == torch.float32 else np.float16)
        self._order = order  # type: ignore[assignment]
        self._voxwid = float(voxwid)
        self._pos_c = np.array(pos_c, dtype=np.float32).reshape(3)
        self._data = t
        return self

    def zeroed_copy(self) -> Volume:
        """A zero-filled volume with this geometry."""
        return Volume.zeros(self._shape, voxwid=self._voxwid, dtype=self._dtype, pos_c=self.pos_c, order=self._order)

    def copy(self) -> Volume:
        """A deep copy."""
        v = self.zeroed_copy()
        v._data.copy_(self._data)
        return v


class FBVolume:
    """A volume given as FORBILD analytic shapes (mirrors volume.py:369-495).

    ``shapes`` is an array of 156-byte FORBILD_Shape records (the reference's
    layout; ``aprict_b200._structs.forbild_shape``). Later shapes override
    earlier ones where they overlap (unless projected in additive mode).
    """

    def __init__(self, shapes: np.ndarray) -> None:
        self.shapes = shapes

    def copy(self) -> FBVolume:
        """A copy of this phantom."""
        return FBVolume(self.shapes.copy())

    def get_bbox(self) -> tuple[np.ndarray, np.ndarray]:
        """(xyz_min, xyz_max) over all shapes (float32)."""
        from .cb import forbild  # noqa: PLC0415

        lo, hi = forbild.shape_bboxes(self.shapes)
        return lo.min(axis=0).astype(np.float32), hi.max(axis=0).astype(np.float32)

    @property
    def minxyz_maxxyz(self) -> tuple[tuple[float, float, float], tuple[float, float, float]]:
        """Bounding box ((minx,miny,minz),(maxx,maxy,maxz))."""
        lo, hi = self.get_bbox()
        return tuple(lo.tolist()), tuple(hi.tolist())  # type: ignore[return-value]

    def prune_to_bbox(self, xyz_min: np.ndarray | tuple, xyz_max: np.ndarray | tuple) -> FBVolume:
        """The shapes whose bounding box meets the given box (volume.py:454-495)."""
        from .cb import forbild  # noqa: PLC0415

        lo, hi = forbild.shape_bboxes(self.shapes)
        bmin = np.asarray(xyz_min, dtype=np.float64)
        bmax = np.asarray(xyz_max, dtype=np.float64)
        keep = np.all(hi >= bmin, axis=1) & np.all(lo <= bmax, axis=1)
        return FBVolume(self.shapes[keep])

    def superimpose_onto(self, vol: FBVolume) -> FBVolume:
        """This phantom's shapes drawn after (over) ``vol``'s."""
        return FBVolume(shapes=np.concatenate((vol.shapes, self.shapes), axis=0))

    # ------------------------------------------------------------- files
    @classmethod
    def load(cls, path_to_pha: str | os.PathLike) -> FBVolume:
        """Read a ``.pha`` phantom file (volume.py:388-390)."""
        from . import pha  # noqa: PLC0415

        return cls(pha.load(path_to_pha))

    @property
    def FORBILD_str(self) -> str:  # noqa: N802
        """The phantom in .pha syntax (volume.py:383-386)."""
        from . import pha  # noqa: PLC0415

        return pha.format_shapes(self.shapes)

    def save(self, path_to_pha: str | os.PathLike) -> None:
        """Write the phantom as a ``.pha`` file (volume.py:392-395)."""
        with open(path_to_pha, mode="w", encoding="utf-8") as f:
            f.write(self.FORBILD_str)

    # ---------------------------------------------------------- sampling
    def to_tensor(
        self,
        xs: np.ndarray,
        ys: np.ndarray,
        zs: np.ndarray,
        *,
        out: torch.Tensor | None = None,
        supersamp_cubic_vox_wid: float | None = None,
        supersamp_factor: int | None = None,
        block: bool = True,
    ) -> torch.Tensor:
        """Point-sample the phantom onto the grid ``xs x ys x zs``, "last shape
        wins", averaging ``supersamp_factor``^3 sub-samples spread over a cube
        of edge ``supersamp_cubic_vox_wid`` per voxel; the result is ADDED to
        ``out`` (float32 CUDA tensor (len(xs), len(ys), len(zs)), new and
        zeroed if None) -- the reference's to_cupy (volume.py:397-418,
        sample_FORBILD_volumes.cu:10-123)."""
        from .cb import forbild  # noqa: PLC0415
        from .cb.flatpanel import _device, _stream  # noqa: PLC0415

        dev = _device()
        axes = [torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev) for a in (xs, ys, zs)]
        shape = tuple(int(a.numel()) for a in axes)
        if out is None:
            out = torch.zeros(shape, dtype=torch.float32, device=dev)
        elif tuple(out.shape) != shape or out.dtype != torch.float32 or not out.is_cuda:
            msg = f"out must be a float32 CUDA tensor of shape {shape}"
            raise ValueError(msg)
        ss = int(supersamp_factor or 1)
        wid = float(supersamp_cubic_vox_wid or 0.0)
        if ss > 1 and wid <= 0.0:
            msg = "supersampling needs supersamp_cubic_vox_wid > 0"
            raise ValueError(msg)
        comp = forbild._compiled(self)  # noqa: SLF001
        if comp.n > 0 and comp.dev is not None:
            _lib.check(
                _lib.lib().aprict_b200_forbild_sample(
                    comp.dev.data_ptr(), comp.n, axes[0].data_ptr(), axes[1].data_ptr(), axes[2].data_ptr(),
                    shape[0], shape[1], shape[2], *out.stride(), out.data_ptr(), wid, ss, _stream(),
                ),
                "forbild_sample",
            )
        if block:
            torch.cuda.current_stream().synchronize()
        return out

    def to_numpy(self, xs: np.ndarray, ys: np.ndarray, zs: np.ndarray, **kw) -> np.ndarray:
        """:meth:`to_tensor` copied to the host (volume.py:503-508)."""
        return self.to_tensor(xs, ys, zs, **kw).cpu().numpy()

    def to_cupy(self, xs: np.ndarray, ys: np.ndarray, zs: np.ndarray, **kw) -> object:
        """:meth:`to_tensor` as a CuPy array (requires CuPy; zero-copy through DLPack)."""
        out = kw.pop("out", None)
        t = self.to_tensor(xs, ys, zs, out=None if out is None else _from_cupy(out), **kw)
        return _to_cupy(t)

    def sample_into(self, volume: Volume, *, supersamp_factor: int = 1) -> Volume:
        """Add the phantom, point-sampled at ``volume``'s voxel centres (with
        ``supersamp_factor``^3 sub-samples per voxel), into ``volume``."""
        xs, ys, zs = volume.xs_ys_zs
        w = volume._f32()  # noqa: SLF001
        self.to_tensor(xs, ys, zs, out=w, supersamp_cubic_vox_wid=volume.voxwid,
                       supersamp_factor=supersamp_factor, block=False)
        volume._commit(w)  # noqa: SLF001
        return volume

    # -------------------------------------------------------- transforms
    _LEN_KEYS = ("x", "y", "z", "r", "l", "dx", "dy", "dz", "r1", "r2")

    def scale_len(self, factor: float) -> None:
        """Scale every length (and clip offset) by ``factor`` (volume.py:510-537)."""
        s = self.shapes.copy()
        for k in self._LEN_KEYS:
            s[k] *= np.float32(factor)
        for c in ("cas1", "cas2", "cas3"):
            s[c]["dotprod"] *= np.float32(factor)
        self.shapes = s

    @staticmethod
    def _axis_name(axis: int | str) -> str:
        names = {0: "x", 1: "y", 2: "z", "x": "x", "y": "y", "z": "z"}
        if axis not in names:
            msg = f"Unknown axis: {axis}"
            raise ValueError(msg)
        return names[axis]

    def flip(self, axis: int | str) -> None:
        """Mirror the phantom along one axis (volume.py:540-573)."""
        a = self._axis_name(axis)
        s = self.shapes.copy()
        s[a] *= -1
        for c in ("cas1", "cas2", "cas3"):
            s[c]["axis"][a] *= -1
        for v in ("axis", "a_x", "a_y", "a_z"):
            s[v][a] *= -1
        self.shapes = s

    def translate(self, axis: int | str, amount: float) -> None:
        """Move the phantom along one axis (volume.py:575-607)."""
        a = self._axis_name(axis)
        s = self.shapes.copy()
        s[a] += np.float32(amount)
        for c in ("cas1", "cas2", "cas3"):
            s[c]["dotprod"] += np.float32(amount) * s[c]["axis"][a]
        self.shapes = s

    def multiply_attenuation(self, amount: float) -> None:
        """Scale every density (volume.py:609-624)."""
        s = self.shapes.copy()
        s["rho"] *= np.float32(amount)
        self.shapes = s


__all__ = ["FBVolume", "Volume"]
