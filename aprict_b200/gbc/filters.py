"""Volume-domain cone-beam ramp filter of the GBC reconstruction (drop-in for
``ramp_filter_conebeam``, src/aprict/gbc/filters.py:256-504).

The reference filters a (x, y, z) volume by rfftn (norm "ortho"), multiplies
the spectrum by |k| / voxel length, divides by the softened Colsher k-factor
of the polar angle from the k_z axis (filters.py:59-147), multiplies by
sinc(f) along each axis, zeroes the DC term and inverts, in about ten array
passes plus the FFTs; then adds a trilinearly upsampled low-resolution
correction. Here: cuFFT for the two transforms (torch.fft), one kernel pass
with every per-frequency factor folded into one FP64 factor
(``aprict_b200_conebeam_spectral``), one kernel pass for the correction
(``aprict_b200_add_upsampled``).
"""

from __future__ import annotations

import logging

import numpy as np
import torch

from .. import _lib


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def ramp_filter_conebeam(
    arr_container: object,
    voxel_phys_len: float,
    cone_angle: float,
    theta_soft: float,
    logger: logging.Logger | None = None,
    log_prefix: str | None = None,  # noqa: ARG001
    allow_overwrite_arr: bool = False,  # noqa: ARG001
    lowres_correction_array: np.ndarray | torch.Tensor | None = None,
    softener: np.ndarray | torch.Tensor | None = None,
    copy_to_array: np.ndarray | torch.Tensor | None = None,
    extra_multiplier: float = 1,
) -> np.ndarray | torch.Tensor:
    """Filter an (n0, n1, n2) volume, axis 2 along the source cylinder's axis.

    ``arr_container`` is the array itself or an object holding it in
    ``.array`` (the reference's NDArrayContainer). A host array gives a host
    result, a CUDA tensor a CUDA tensor (or the filled ``copy_to_array``).
    """
    arr = getattr(arr_container, "array", arr_container)
    if logger is not None and cone_angle == 0:
        logger.warning("ramp_filter_conebeam has been supplied with cone_angle = 0. This is not intended use.")
    if cone_angle < 0:
        msg = f"Cone angle is negative: {cone_angle}"
        raise ValueError(msg)
    if cone_angle > np.pi:
        msg = f"Cone angle greater than pi: {cone_angle}"
        raise ValueError(msg)
    host = isinstance(arr, np.ndarray)
    x = torch.as_tensor(np.ascontiguousarray(arr, dtype=np.float32) if host else arr)
    if x.dim() != 3:
        msg = "ramp_filter_conebeam filters a 3-D volume"
        raise ValueError(msg)
    x = x.to(device="cuda", dtype=torch.float32)
    n0, n1, n2 = (int(s) for s in x.shape)
    factor = None
    if lowres_correction_array is not None:
        low = lowres_correction_array
        sl = tuple(int(s) for s in low.shape)
        if any(a % b for a, b in zip((n0, n1, n2), sl)):
            msg = "The provided lowres_correction_array shape does not divide into the full array shape."
            raise ValueError(msg)
        fs = {a // b for a, b in zip((n0, n1, n2), sl)}
        if len(fs) != 1:
            msg = "The provided lowres_correction_array shape does not divide evenly into the full array shape."
            raise ValueError(msg)
        factor = fs.pop()
    if copy_to_array is not None and tuple(copy_to_array.shape) != (n0, n1, n2):
        msg = "Output array does not match the shape of the input array."
        raise ValueError(msg)

    spec = torch.fft.rfftn(x, norm="ortho").contiguous()
    _lib.check(
        _lib.lib().aprict_b200_conebeam_spectral(
            spec.data_ptr(), n0, n1, n2, float(extra_multiplier) / float(voxel_phys_len), float(cone_angle),
            float(theta_soft), _stream(),
        ),
        "conebeam_spectral",
    )
    out = torch.fft.irfftn(spec, s=(n0, n1, n2), norm="ortho").contiguous()
    del spec
    if factor is not None:
        low = torch.as_tensor(lowres_correction_array).to(device="cuda", dtype=torch.float32).contiguous()
        _lib.check(
            _lib.lib().aprict_b200_add_upsampled(
                out.data_ptr(), n0, n1, n2, low.data_ptr(), *(int(s) for s in low.shape), int(factor), _stream()
            ),
            "add_upsampled",
        )
    if softener is not None:
        out *= torch.as_tensor(softener).to(device="cuda", dtype=torch.float32)
    if copy_to_array is not None:
        if isinstance(copy_to_array, np.ndarray):
            copy_to_array[...] = out.cpu().numpy()
        else:
            copy_to_array.copy_(out)
        return copy_to_array
    return out.cpu().numpy() if host else out


__all__ = ["ramp_filter_conebeam"]
