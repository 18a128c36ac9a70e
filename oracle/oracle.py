"""ctypes front for the parity oracles.

TEST INFRASTRUCTURE ONLY -- the checker. Imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline / reference arm; the
aprict_b200 package never imports it and no product path calls it.

Two libraries, both built by oracle/Makefile:
  * liboracle.so -- our FP64 restatement of the reference's arithmetic
    (ab_oracle.c; citations there);
  * _ref/libaprict_ref.so -- the reference's own device code
    (src/aprict/data/cusrc/CB_project_texture_chunked.cu, CB_backproject.cu,
    FORBILD_volumes.h) compiled for the CPU in place from the reference
    checkout. It exists only where the reference sources were present at build
    time; ``have_ref()`` says whether it was built.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libaprict_ref.so"

proj_spec = np.dtype(
    {
        "names": ["source_pos", "det_pos", "det_u", "det_v", "nu", "nv", "type"],
        "formats": [np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4")])] * 4 + ["<u4", "<u4", "u1"],
        "offsets": [0, 12, 24, 36, 48, 52, 56],
        "itemsize": 60,
    }
)


class AoGrid(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int),
        ("ny", ctypes.c_int),
        ("nz", ctypes.c_int),
        ("order", ctypes.c_int),
        ("voxwid", ctypes.c_double),
        ("corner", ctypes.c_double * 3),
    ]


class AoBpCfg(ctypes.Structure):
    _fields_ = [
        ("exact", ctypes.c_int),
        ("all_ones", ctypes.c_int),
        ("mask", ctypes.c_int),
        ("mask_rad", ctypes.c_double),
        ("sep", ctypes.c_double),
        ("pL", ctypes.c_int),
        ("pV", ctypes.c_int),
        ("val", ctypes.c_double),
        ("raycast", ctypes.c_int),
        ("linear", ctypes.c_int),
        ("ssx", ctypes.c_int),
        ("ssy", ctypes.c_int),
        ("ssz", ctypes.c_int),
        ("preset", ctypes.c_int),
    ]


def build(ref_dir: pathlib.Path | str | None = None, *, quiet: bool = True) -> None:
    """Build liboracle.so, and _ref/libaprict_ref.so when the reference sources exist.

    ``ref_dir`` (or the APRICT_REF_DIR environment variable) names the reference
    checkout; without either, the Makefile's default location is used.
    """
    cmd = ["make", "-C", str(HERE), "liboracle.so", "ref-if-present"]
    if ref_dir is not None:
        cmd.append(f"REF={ref_dir}")
    out = subprocess.run(cmd, capture_output=True, text=True, check=False)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_so: dict[str, ctypes.CDLL] = {}


def _load(path: pathlib.Path) -> ctypes.CDLL:
    key = str(path)
    if key not in _so:
        if not path.exists():
            msg = f"{path} is not built (run `make -C oracle`)"
            raise RuntimeError(msg)
        _so[key] = ctypes.CDLL(key)
    return _so[key]


def have_ref() -> bool:
    """Whether the reference-compiled library is available."""
    return REF_SO.exists()


def nthreads_default() -> int:
    return int(os.environ.get("APRICT_ORACLE_THREADS", "0")) or (os.cpu_count() or 1)


def _p(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def grid(shape: tuple[int, int, int], voxwid: float, corner: np.ndarray, order: str = "C") -> AoGrid:
    g = AoGrid()
    g.nx, g.ny, g.nz = (int(s) for s in shape)
    g.order = 0 if order == "C" else 1
    g.voxwid = float(np.float32(voxwid))
    for i in range(3):
        g.corner[i] = float(np.float32(corner[i]))
    return g


def _specs(specs: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(specs.reshape(-1))
    if s.dtype.itemsize != 60:
        msg = "specs must be 60-byte proj_spec records"
        raise ValueError(msg)
    return s


def _vol_flat(vol: np.ndarray, order: str) -> np.ndarray:
    return np.ascontiguousarray(vol.astype(np.float32)) if order == "C" else np.asfortranarray(vol.astype(np.float32))


# ----------------------------------------------------------------------- FP64 oracle
def project_siddon(
    specs: np.ndarray,
    vol: np.ndarray,
    *,
    voxwid: float,
    corner: np.ndarray,
    order: str = "C",
    svf: float = 1.0,
    mba: float = 1.0,
    ssu: int = 1,
    ssv: int = 1,
    nthreads: int | None = None,
) -> tuple[np.ndarray, int]:
    """FP64 Siddon projection; returns (out (M,nu,nv) float64, number of ray-voxel segments)."""
    lib = _load(ORACLE_SO)
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    v = _vol_flat(vol, order)
    out = np.zeros((m, nu, nv), dtype=np.float64)
    nseg = ctypes.c_int64(0)
    g = grid(vol.shape, voxwid, corner, order)
    lib.ao_project_siddon(
        _p(s), m, nu, nv, _p(v), ctypes.byref(g), ctypes.c_double(svf), ctypes.c_double(mba), ssu, ssv, _p(out),
        ctypes.byref(nseg), nthreads or nthreads_default(),
    )
    return out, int(nseg.value)


def backproject_transpose(
    specs: np.ndarray,
    projs: np.ndarray,
    shape: tuple[int, int, int],
    *,
    voxwid: float,
    corner: np.ndarray,
    order: str = "C",
    svf: float = 1.0,
    mba: float = 1.0,
    ssu: int = 1,
    ssv: int = 1,
    nthreads: int | None = None,
) -> np.ndarray:
    """FP64 transpose of :func:`project_siddon` (returns a volume in ``order``)."""
    lib = _load(ORACLE_SO)
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    p = np.ascontiguousarray(projs, dtype=np.float64)
    out = np.zeros(shape, dtype=np.float64, order=order)
    g = grid(shape, voxwid, corner, order)
    lib.ao_backproject_transpose(
        _p(s), m, nu, nv, _p(p), ctypes.byref(g), ctypes.c_double(svf), ctypes.c_double(mba), ssu, ssv, _p(out),
        nthreads or nthreads_default(),
    )
    return out


def bp_cfg_from_contents(c: np.ndarray) -> AoBpCfg:
    """Oracle config from a packed aprict_backproject_config record."""
    k = AoBpCfg()
    k.exact = int(c["exact"])
    k.all_ones = int(c["backproject_all_1s"])
    k.mask = int(c["mask_to_cylinder"])
    k.mask_rad = float(c["mask_to_cyl_rad"])
    k.sep = float(c["soften_edge_proportion"])
    k.pL = int(c["Z_on_L_factor_power"])
    k.pV = int(c["Z_on_val_factor_power"])
    k.val = float(c["Z_on_val_factor_val"])
    k.raycast = int(c["approx_mode_direct_raycast"])
    k.linear = int(c["approx_mode_linear_interpolate"])
    k.preset = int(c["weighting_preset"])
    k.ssx, k.ssy, k.ssz = int(c["ssx"]), int(c["ssy"]), int(c["ssz"])
    return k


def backproject(
    specs: np.ndarray,
    projs: np.ndarray,
    shape: tuple[int, int, int],
    cfg_contents: np.ndarray,
    *,
    voxwid: float,
    corner: np.ndarray,
    order: str = "C",
    mult: np.ndarray | None = None,
    nthreads: int | None = None,
) -> np.ndarray:
    """FP64 voxel-driven backprojection (returns the increment, a volume in ``order``)."""
    lib = _load(ORACLE_SO)
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    p = np.ascontiguousarray(projs, dtype=np.float64)
    out = np.zeros(shape, dtype=np.float64, order=order)
    g = grid(shape, voxwid, corner, order)
    k = bp_cfg_from_contents(cfg_contents)
    mm = None if mult is None else np.asarray(mult, dtype=np.float64, order=order)
    lib.ao_backproject(
        _p(s), m, nu, nv, _p(p), ctypes.byref(g), None if mm is None else _p(mm), ctypes.byref(k), _p(out),
        nthreads or nthreads_default(),
    )
    return out


def bp_nearest_ties(
    specs: np.ndarray,
    shape: tuple[int, int, int],
    cfg_contents: np.ndarray,
    *,
    voxwid: float,
    corner: np.ndarray,
    order: str = "C",
    eps: float = 1e-9,
    nthreads: int | None = None,
) -> np.ndarray:
    """Per voxel, the number of fast-nearest (sub-sample, view) pairs whose pixel choice
    lies within eps pixel of a half-integer tie (FP64 cannot settle those)."""
    lib = _load(ORACLE_SO)
    s = _specs(specs)
    out = np.zeros(shape, dtype=np.int32, order=order)
    g = grid(shape, voxwid, corner, order)
    k = bp_cfg_from_contents(cfg_contents)
    lib.ao_bp_nearest_ties(_p(s), len(s), ctypes.byref(g), ctypes.byref(k), ctypes.c_double(eps), _p(out),
                           nthreads or nthreads_default())
    return out


# ------------------------------------------------------- reference compiled for the CPU
def ref_project_siddon(
    specs: np.ndarray,
    vol: np.ndarray,
    *,
    voxwid: float,
    corner: np.ndarray,
    svf: float = 1.0,
    mba: float = 1.0,
    ssu: int = 1,
    ssv: int = 1,
    out: np.ndarray | None = None,
    nthreads: int | None = None,
) -> np.ndarray:
    """The reference's project_CB_texture_chunked<float,float> run on the CPU (C-order volume)."""
    lib = _load(REF_SO)
    lib.ref_project_siddon.restype = ctypes.c_longlong
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    v = np.ascontiguousarray(vol, dtype=np.float32)
    o = np.zeros((m, nu, nv), dtype=np.float32) if out is None else out
    tp = np.asarray(corner, dtype=np.float32)
    oob = lib.ref_project_siddon(
        _p(s), m, nu, nv, _p(v), vol.shape[0], vol.shape[1], vol.shape[2], ctypes.c_float(voxwid), _p(tp),
        ctypes.c_float(svf), ctypes.c_float(mba), ssu, ssv, _p(o), nthreads or nthreads_default(),
    )
    if oob:
        msg = f"reference projector read outside the volume {oob} times"
        raise RuntimeError(msg)
    return o


def ref_backproject(
    specs: np.ndarray,
    projs: np.ndarray,
    vol: np.ndarray,
    cfg_contents: np.ndarray,
    *,
    voxwid: float,
    corner: np.ndarray,
    mult: np.ndarray | None = None,
    nthreads: int | None = None,
) -> np.ndarray:
    """The reference's backproject_CB_voltex<float,float> on the CPU; accumulates into ``vol`` (C order float32)."""
    lib = _load(REF_SO)
    lib.ref_backproject.restype = ctypes.c_longlong
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    p = np.ascontiguousarray(projs, dtype=np.float32)
    if not (vol.flags["C_CONTIGUOUS"] and vol.dtype == np.float32):
        msg = "vol must be a C-contiguous float32 array"
        raise ValueError(msg)
    mm = None if mult is None else np.ascontiguousarray(mult, dtype=np.float32)
    c = cfg_contents
    tp = np.asarray(corner, dtype=np.float32)
    f = ctypes.c_float
    oob = lib.ref_backproject(
        _p(s), m, nu, nv, _p(p), _p(vol), vol.shape[0], vol.shape[1], vol.shape[2], f(voxwid), _p(tp),
        None if mm is None else _p(mm), int(c["exact"]), int(c["backproject_all_1s"]), int(c["mask_to_cylinder"]),
        f(float(c["mask_to_cyl_rad"])), f(float(c["soften_edge_proportion"])), int(c["Z_on_L_factor_power"]),
        int(c["Z_on_val_factor_power"]), f(float(c["Z_on_val_factor_val"])), int(c["approx_mode_direct_raycast"]),
        int(c["approx_mode_linear_interpolate"]), int(c["ssx"]), int(c["ssy"]), int(c["ssz"]), int(c["weighting_preset"]),
        nthreads or nthreads_default(),
    )
    if oob:
        msg = f"reference backprojector accessed outside the volume {oob} times"
        raise RuntimeError(msg)
    return vol


def ref_backproject_gbc(
    specs: np.ndarray,
    projs: np.ndarray,
    vol: np.ndarray,
    vol2: np.ndarray,
    cfg_contents: np.ndarray,
    *,
    voxwid: float,
    corner: np.ndarray,
    mult: np.ndarray | None = None,
    nthreads: int | None = None,
) -> tuple[np.ndarray, np.ndarray]:
    """The reference's backproject_CB_voltex_GBC_cyl<float,float> on the CPU; accumulates into
    ``vol`` and the weight sums into ``vol2`` (both C order float32)."""
    lib = _load(REF_SO)
    lib.ref_backproject_gbc.restype = ctypes.c_longlong
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    p = np.ascontiguousarray(projs, dtype=np.float32)
    for v in (vol, vol2):
        if not (v.flags["C_CONTIGUOUS"] and v.dtype == np.float32):
            msg = "volumes must be C-contiguous float32 arrays"
            raise ValueError(msg)
    mm = None if mult is None else np.ascontiguousarray(mult, dtype=np.float32)
    c = cfg_contents
    soft = np.array([c["soft_vartheta_v"], c["soft_vartheta_v_softspan"], c["soft_vartheta_h"],
                     c["soft_vartheta_h_softspan"]], dtype=np.float32)
    tp = np.asarray(corner, dtype=np.float32)
    f = ctypes.c_float
    oob = lib.ref_backproject_gbc(
        _p(s), m, nu, nv, _p(p), _p(vol), _p(vol2), vol.shape[0], vol.shape[1], vol.shape[2], f(voxwid), _p(tp),
        None if mm is None else _p(mm), f(float(c["Z_on_val_factor_val"])), int(c["approx_mode_linear_interpolate"]),
        int(c["ssx"]), int(c["ssy"]), int(c["ssz"]), _p(soft), nthreads or nthreads_default(),
    )
    if oob:
        msg = f"reference GBC backprojector accessed outside the volume {oob} times"
        raise RuntimeError(msg)
    return vol, vol2


def ref_gbc_weight(R: float, vox: np.ndarray, src: np.ndarray, soft: np.ndarray) -> np.ndarray:  # noqa: N803
    """The reference's _GBC_weightfun<float> at points vox (n, 3) for sources src (n, 3);
    soft = (vartheta_v, span_v, vartheta_h, span_h)."""
    lib = _load(REF_SO)
    v = np.ascontiguousarray(vox, dtype=np.float32)
    s = np.ascontiguousarray(src, dtype=np.float32)
    so = np.ascontiguousarray(soft, dtype=np.float32)
    out = np.empty(len(v), np.float32)
    lib.ref_gbc_weight(ctypes.c_float(R), _p(v), _p(s), _p(so), ctypes.c_longlong(len(v)), _p(out))
    return out


# --------------------------------------------------------------------- FORBILD shapes
def project_forbild(
    specs: np.ndarray,
    shapes: np.ndarray,
    *,
    mba: float = 1.0,
    mode: int = 0,
    ssu: int = 1,
    ssv: int = 1,
    nthreads: int | None = None,
) -> np.ndarray:
    """FP64 analytic projection of FORBILD shapes; mode 0 later-wins, 1 sum rho dt, 2 sum rho dt |seg|."""
    lib = _load(ORACLE_SO)
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    sh = np.ascontiguousarray(shapes.reshape(-1))
    out = np.zeros((m, nu, nv), dtype=np.float64)
    lib.ao_project_forbild(
        _p(s), m, nu, nv, _p(sh), len(sh), ctypes.c_double(mba), mode, ssu, ssv, _p(out), nthreads or nthreads_default()
    )
    return out


def forbild_interval(v1: np.ndarray, v2: np.ndarray, shape: np.ndarray) -> tuple[float, float] | None:
    """FP64 interval of segment v1->v2 with one shape (None if empty)."""
    lib = _load(ORACLE_SO)
    a = np.asarray(v1, np.float64)
    b = np.asarray(v2, np.float64)
    o = np.zeros(2)
    sh = np.ascontiguousarray(shape.reshape(1))
    ok = lib.ao_forbild_interval(_p(a), _p(b), _p(sh), _p(o))
    return (float(o[0]), float(o[1])) if ok else None


def ref_project_forbild(
    specs: np.ndarray,
    shapes: np.ndarray,
    *,
    mba: float = 1.0,
    overlap_addition: bool = False,
    ssu: int = 1,
    ssv: int = 1,
    nthreads: int | None = None,
) -> tuple[np.ndarray, int]:
    """The reference's FORBILD projection body run on the CPU: (out float32, overflow count)."""
    lib = _load(REF_SO)
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    sh = np.ascontiguousarray(shapes.reshape(-1))
    out = np.zeros((m, nu, nv), dtype=np.float32)
    ovf = ctypes.c_uint(0)
    lib.ref_project_forbild(
        _p(s), m, nu, nv, _p(sh), len(sh), ctypes.c_float(mba), int(overlap_addition), ssu, ssv, _p(out),
        ctypes.byref(ovf), nthreads or nthreads_default(),
    )
    return out, int(ovf.value)


def ref_forbild_interval(v1: np.ndarray, v2: np.ndarray, shape: np.ndarray) -> tuple[float, float]:
    """The reference's FORBILD_clip_line_segment(FORBILD_Shape) on the CPU (FP32)."""
    lib = _load(REF_SO)
    a = np.asarray(v1, np.float32)
    b = np.asarray(v2, np.float32)
    o = np.zeros(2, np.float32)
    sh = np.ascontiguousarray(shape.reshape(1))
    lib.ref_forbild_interval(_p(a), _p(b), _p(sh), _p(o))
    return float(o[0]), float(o[1])


def forbild_sample(shapes: np.ndarray, xs, ys, zs, *, ss_wid: float = 0.0, ss: int = 1,
                   nthreads: int | None = None) -> np.ndarray:
    """FP64 "last shape wins" point sampling (natural-coordinate point tests)."""
    lib = _load(ORACLE_SO)
    ax = [np.ascontiguousarray(a, np.float64) for a in (xs, ys, zs)]
    sh = np.ascontiguousarray(shapes.reshape(-1))
    out = np.zeros((len(ax[0]), len(ax[1]), len(ax[2])), np.float64)
    lib.ao_forbild_sample(_p(sh), len(sh), _p(ax[0]), _p(ax[1]), _p(ax[2]), len(ax[0]), len(ax[1]), len(ax[2]),
                          ctypes.c_double(ss_wid), ss, _p(out), nthreads or nthreads_default())
    return out


def ref_forbild_sample(shapes: np.ndarray, xs, ys, zs, *, ss_wid: float = 0.0, ss: int = 1,
                       nthreads: int | None = None) -> np.ndarray:
    """The reference's sampling body (its own _in_region, FP32) on the CPU."""
    lib = _load(REF_SO)
    ax = [np.ascontiguousarray(a, np.float32) for a in (xs, ys, zs)]
    sh = np.ascontiguousarray(shapes.reshape(-1))
    out = np.zeros((len(ax[0]), len(ax[1]), len(ax[2])), np.float32)
    lib.ref_forbild_sample(_p(sh), len(sh), _p(ax[0]), _p(ax[1]), _p(ax[2]), len(ax[0]), len(ax[1]), len(ax[2]),
                           ctypes.c_float(ss_wid), ss, _p(out), nthreads or nthreads_default())
    return out


# ------------------------------------------------------- reference kernels on the GPU
REF_GPU_SO = HERE / "_ref" / "libaprict_refgpu.so"


def have_ref_gpu() -> bool:
    """Whether the reference's GPU kernels were built (oracle/_ref/libaprict_refgpu.so)."""
    return REF_GPU_SO.exists()


class RefGpuVolume:
    """A C-order float32 volume in a CUDA array behind a surface object, as the
    reference's Texture holds it; the reference's own kernels read and write it.

    ``src`` is a CUDA float32 tensor of shape (nx, ny, nz), C-contiguous."""

    def __init__(self, src) -> None:  # noqa: ANN001
        self._lib = _load(REF_GPU_SO)
        self._lib.refgpu_vol_destroy.restype = None
        nx, ny, nz = (int(s) for s in src.shape)
        if not (src.is_cuda and src.is_contiguous() and str(src.dtype) == "torch.float32"):
            msg = "the volume must be a C-contiguous float32 CUDA tensor"
            raise ValueError(msg)
        self.shape = (nx, ny, nz)
        h = ctypes.c_void_p()
        rc = self._lib.refgpu_vol_create(ctypes.c_void_p(src.data_ptr()), nx, ny, nz, ctypes.byref(h))
        if rc != 0:
            msg = f"refgpu_vol_create failed with CUDA error {rc}"
            raise RuntimeError(msg)
        self.handle = h

    def read(self, dst, stream: int = 0) -> None:  # noqa: ANN001
        _check_cuda(self._lib.refgpu_vol_read(self.handle, ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(stream)),
                    "refgpu_vol_read")

    def write(self, src, stream: int = 0) -> None:  # noqa: ANN001
        _check_cuda(self._lib.refgpu_vol_write(self.handle, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(stream)),
                    "refgpu_vol_write")

    def close(self) -> None:
        if self.handle:
            self._lib.refgpu_vol_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # noqa: BLE001, S110
            pass


def _check_cuda(rc: int, what: str) -> None:
    if rc != 0:
        msg = f"{what} failed with CUDA error {rc}"
        raise RuntimeError(msg)


def ref_gpu_project(vol: RefGpuVolume, specs_dev, n_views: int, nu: int, nv: int, out, *, voxwid: float,  # noqa: ANN001
                    corner: np.ndarray, svf: float = 1.0, mba: float = 1.0, ssu: int = 1, ssv: int = 1,
                    stream: int = 0) -> None:
    """The reference's project_CB_texture_chunked<float,float>, launched as flatpanel.project
    launches it; accumulates into ``out`` (a C-contiguous (n_views, nu, nv) float32 CUDA tensor)."""
    lib = _load(REF_GPU_SO)
    tp = np.asarray(corner, dtype=np.float32)
    f = ctypes.c_float
    _check_cuda(lib.refgpu_project(vol.handle, f(voxwid), _p(tp), ctypes.c_void_p(specs_dev), n_views, nu, nv,
                                   ctypes.c_void_p(out.data_ptr()), f(svf), f(mba), ssu, ssv, ctypes.c_void_p(stream)),
                "refgpu_project")


def ref_gpu_backproject(vol: RefGpuVolume, specs: np.ndarray, projs, cfg_contents: np.ndarray, *,  # noqa: ANN001
                        voxwid: float, corner: np.ndarray, mult: RefGpuVolume | None = None, stream: int = 0) -> None:
    """The reference's backproject_CB_voltex<float,float>, launched as flatpanel.backproject
    launches it (one launch per 10 views); adds into ``vol``. ``projs``: a C-contiguous
    (n_views, nu, nv) float32 CUDA tensor; ``specs``: the host proj_spec records."""
    lib = _load(REF_GPU_SO)
    s = _specs(specs)
    m, nu, nv = len(s), int(s["nu"][0]), int(s["nv"][0])
    c = cfg_contents
    if int(c["weighting_preset"]) != 0:
        msg = "ref_gpu_backproject runs weighting preset 0 only"
        raise ValueError(msg)
    tp = np.asarray(corner, dtype=np.float32)
    f = ctypes.c_float
    _check_cuda(lib.refgpu_backproject(
        vol.handle, None if mult is None else mult.handle, f(voxwid), _p(tp), _p(s), m, nu, nv,
        ctypes.c_void_p(projs.data_ptr()), int(c["exact"]), int(c["backproject_all_1s"]), int(c["mask_to_cylinder"]),
        f(float(c["mask_to_cyl_rad"])), f(float(c["soften_edge_proportion"])), int(c["Z_on_L_factor_power"]),
        int(c["Z_on_val_factor_power"]), f(float(c["Z_on_val_factor_val"])), int(c["approx_mode_direct_raycast"]),
        int(c["approx_mode_linear_interpolate"]), int(c["ssx"]), int(c["ssy"]), int(c["ssz"]),
        ctypes.c_void_p(stream)), "refgpu_backproject")
