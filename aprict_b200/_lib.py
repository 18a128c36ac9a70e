"""ctypes binding of libaprict_b200.so (the C ABI declared in include/aprict_b200.h).

The library is the only compute path: if it is missing or fails to load,
:func:`lib` raises, and no operator falls back to another implementation.
"""

from __future__ import annotations

import ctypes
import pathlib
import threading

import numpy as np

from . import _structs as S

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libaprict_b200.so"

# Every symbol declared in include/aprict_b200.h, with its ctypes signature.
_c_int, _c_void_p, _c_char_p = ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p
SIGNATURES: dict[str, tuple[object, list[object]]] = {
    "aprict_b200_status_string": (_c_char_p, [_c_int]),
    "aprict_b200_last_error": (_c_char_p, []),
    "aprict_b200_version": (_c_char_p, []),
    "aprict_b200_struct_size": (ctypes.c_size_t, [_c_char_p]),
    "aprict_b200_set_tuning": (_c_int, [_c_int, _c_int]),
    "aprict_b200_get_tuning": (_c_int, [_c_int]),
    "aprict_b200_project_siddon": (
        _c_int,
        [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p],
    ),
    "aprict_b200_backproject_scatter": (
        _c_int,
        [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p],
    ),
    "aprict_b200_backproject": (
        _c_int,
        [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p],
    ),
    "aprict_b200_vol_fill": (_c_int, [_c_void_p, ctypes.c_int64, ctypes.c_float, _c_void_p]),
    "aprict_b200_vol_scale": (_c_int, [_c_void_p, ctypes.c_int64, ctypes.c_float, _c_void_p]),
    "aprict_b200_vol_invert": (_c_int, [_c_void_p, ctypes.c_int64, _c_int, ctypes.c_float, _c_void_p]),
    "aprict_b200_vol_softmask_cylinder": (_c_int, [_c_void_p, _c_void_p, ctypes.c_float, _c_void_p]),
    "aprict_b200_vol_dot": (_c_int, [_c_void_p, _c_void_p, ctypes.c_int64, _c_void_p, _c_void_p]),
    "aprict_b200_vol_mul": (_c_int, [_c_void_p, _c_void_p, _c_void_p, ctypes.c_int64, _c_void_p]),
    "aprict_b200_vol_axpy": (
        _c_int,
        [_c_void_p, _c_void_p, ctypes.c_float, _c_void_p, ctypes.c_int64, _c_void_p],
    ),
    "aprict_b200_ramp_filter": (
        _c_int,
        [
            _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_int, _c_void_p,
            ctypes.c_int64, ctypes.c_int64, ctypes.c_float, _c_void_p,
        ],
    ),
    "aprict_b200_ramp_fft_tables_bytes": (ctypes.c_int64, [ctypes.c_int64]),
    "aprict_b200_ramp_fft_tables": (_c_int, [_c_void_p, ctypes.c_int64, _c_void_p, _c_void_p]),
    "aprict_b200_ramp_filter_fft": (
        _c_int,
        [
            _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
            ctypes.c_int64, ctypes.c_int64, ctypes.c_float, _c_void_p,
        ],
    ),
    "aprict_b200_vol_div_softzero": (
        _c_int, [_c_void_p, _c_void_p, _c_void_p, ctypes.c_int64, ctypes.c_float, _c_void_p],
    ),
    "aprict_b200_vol_mul_xygrid": (_c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p]),
    "aprict_b200_backproject_gbc": (
        _c_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                 _c_void_p],
    ),
    "aprict_b200_gbc_weight_integral": (
        _c_int, [_c_void_p, ctypes.c_int32, _c_void_p, ctypes.c_int32, ctypes.c_int32, _c_void_p, _c_void_p],
    ),
    "aprict_b200_conebeam_spectral": (
        _c_int, [_c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                 ctypes.c_double, _c_void_p],
    ),
    "aprict_b200_add_upsampled": (
        _c_int, [_c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _c_void_p, ctypes.c_int32, ctypes.c_int32,
                 ctypes.c_int32, ctypes.c_int32, _c_void_p],
    ),
    "aprict_b200_rotate_projections": (
        _c_int,
        [
            _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, ctypes.c_double, ctypes.c_double,
            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _c_void_p, _c_void_p, _c_void_p,
        ],
    ),
    "aprict_b200_forbild_compile": (_c_int, [_c_void_p, ctypes.c_int64, _c_void_p]),
    "aprict_b200_forbild_sample": (
        _c_int,
        [_c_void_p, ctypes.c_int64, _c_void_p, _c_void_p, _c_void_p, ctypes.c_uint32, ctypes.c_uint32,
         ctypes.c_uint32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _c_void_p, ctypes.c_float,
         ctypes.c_uint32, _c_void_p],
    ),
    "aprict_b200_sirt_step": (_c_int, [_c_void_p] * 9 + [_c_void_p]),
    "aprict_b200_sirt_graph_create": (_c_int, [_c_void_p] * 9 + [_c_int, _c_void_p]),
    "aprict_b200_sirt_graph_launch": (_c_int, [_c_void_p, _c_void_p]),
    "aprict_b200_sirt_graph_iterations": (_c_int, [_c_void_p]),
    "aprict_b200_sirt_graph_destroy": (None, [_c_void_p]),
    "aprict_b200_batch_plan_bytes": (ctypes.c_size_t, [_c_int, _c_int]),
    "aprict_b200_batch_plan": (_c_int, [_c_int, _c_void_p, _c_int, _c_void_p, _c_void_p, ctypes.c_size_t]),
    "aprict_b200_batch_run": (_c_int, [_c_void_p, _c_void_p, _c_void_p]),
    "aprict_b200_batch_run_static": (_c_int, [_c_void_p, _c_void_p]),
    "aprict_b200_project_forbild": (
        _c_int,
        [
            _c_void_p, _c_void_p, _c_void_p, _c_void_p, ctypes.c_int64, ctypes.c_float, ctypes.c_uint32,
            ctypes.c_uint32, _c_int, _c_void_p, _c_void_p, _c_void_p,
        ],
    ),
}

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


class AprictError(RuntimeError):
    """A nonzero aprict_status returned by the C ABI."""

    def __init__(self, status: int, where: str, detail: str) -> None:
        self.status = status
        super().__init__(f"{where}: {detail} (status {status})")


def lib() -> ctypes.CDLL:
    """Load (once) and return the shared library; raise if it is unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                msg = f"{LIB_PATH.name} is not built; run `python -m aprict_b200.build`"
                raise RuntimeError(msg)
            handle = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def check(status: int, where: str) -> None:
    """Raise the exception class the reference raises for the same condition."""
    if status == 0:
        return
    detail = lib().aprict_b200_last_error().decode() or lib().aprict_b200_status_string(status).decode()
    if status == 1:
        raise ValueError(f"{where}: {detail}")
    if status == 2:
        raise NotImplementedError(f"{where}: {detail}")
    raise AprictError(status, where, detail)


def upload(a: np.ndarray):  # noqa: ANN201
    """A copy of host array ``a`` on the current CUDA device, enqueued on the
    current stream without blocking the host.

    A plain copy from pageable memory waits for the stream to drain first, so
    the GPU would idle while the host prepares the next launch; here ``a`` is
    staged in pinned memory (torch's caching host allocator holds the block
    until the copy has run) and copied asynchronously. ``a`` may be changed
    or freed as soon as this returns."""
    import torch  # noqa: PLC0415

    host = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return host.to(torch.device("cuda", torch.cuda.current_device()), non_blocking=True)


def ptr(a: np.ndarray) -> ctypes.c_void_p:
    """Pointer to a numpy array's data (struct arguments are passed by
    pointer). The pointer object holds a reference to the array, so a
    temporary array stays alive for the duration of the call it is passed to."""
    return a.ctypes.data_as(ctypes.c_void_p)


def vol_desc(shape: tuple[int, int, int], order: str, voxwid: float, corner: np.ndarray) -> np.ndarray:
    d = np.zeros((), dtype=S.vol_desc)
    d["nx"], d["ny"], d["nz"] = shape
    d["order"] = 0 if order == "C" else 1
    d["voxwid"] = np.float32(voxwid)
    d["corner"] = tuple(np.asarray(corner, dtype=np.float32).tolist())
    return d


def proj_desc(shape: tuple[int, int, int], strides: tuple[int, int, int]) -> np.ndarray:
    d = np.zeros((), dtype=S.proj_desc)
    d["n_views"], d["nu"], d["nv"] = shape
    d["stride_view"], d["stride_u"], d["stride_v"] = strides
    return d
