"""Expected sum of GBC backprojection weights over a perfect cylindrical
source locus (drop-in for src/aprict/gbc/weightinteg.py:22-91).

The integral over source heights and angles is evaluated by
``aprict_b200_gbc_weight_integral`` (one thread per (height, angle) sample,
FP64 block sums); the xy-grid form interpolates it linearly in the radius.
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _lib
from ..cb import flatpanel as cbfp


def backproj_gbc_weight_integ_GPU(  # noqa: N802
    r_on_R: np.ndarray,  # noqa: N803
    config: cbfp.ConfigBackproject,
    num_z_samps: int,
    num_ang_samps: int,
) -> np.ndarray:
    """The integrated weight x softening at each radius ``r_on_R`` (units of R, 1-D, increasing)."""
    r_on_R = np.asarray(r_on_R)  # noqa: N806
    if r_on_R.ndim != 1:
        msg = "r_on_R should be a 1-dimensional array."
        raise ValueError(msg)
    r = torch.from_numpy(np.ascontiguousarray(r_on_R, dtype=np.float32)).cuda()
    out = torch.zeros(len(r_on_R), dtype=torch.float64, device="cuda")
    cfg = config.contents
    _lib.check(
        _lib.lib().aprict_b200_gbc_weight_integral(
            r.data_ptr(), len(r_on_R), out.data_ptr(), int(num_z_samps), int(num_ang_samps), _lib.ptr(cfg),
            torch.cuda.current_stream().cuda_stream,
        ),
        "gbc_weight_integral",
    )
    return out.cpu().numpy().astype(np.float32)


def backproj_gbc_weight_integ_xygrid_GPU(  # noqa: N802
    xs: np.ndarray,
    ys: np.ndarray,
    R: float,  # noqa: N803
    config: cbfp.ConfigBackproject,
    num_z_samps: int = 6000,
    num_ang_samps: int = 6000,
) -> np.ndarray:
    """The integrated weights on the (len(xs), len(ys)) grid of voxel centres."""
    rel = np.sqrt(np.square(xs[:, np.newaxis]) + np.square(ys[np.newaxis, :])) / R
    numsamps = 2 * max(len(xs), len(ys))
    r_in = np.linspace(rel.min(), rel.max(), endpoint=True, num=numsamps)
    integ = backproj_gbc_weight_integ_GPU(r_in, config, num_z_samps, num_ang_samps)
    return np.interp(rel, r_in, integ)


__all__ = ["backproj_gbc_weight_integ_GPU", "backproj_gbc_weight_integ_xygrid_GPU"]
