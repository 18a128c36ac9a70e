"""Landweber iteration on the GPU (drop-in for ``aprict.iterators.Landweber_flatpanel``).

Follows src/aprict/iterators/landweber_vram.py:35-265: for each ordered
subset k, x <- x + (accel / rho_k) B (b_k - A x), with rho_k the Rayleigh
quotient of B A estimated by ``rayleigh_quotient_num_iterations`` power
iterations from a random positive volume (:127-209), and B the fast
backprojector with a cylinder mask and a detector-edge taper (:104-109).
``exact_adjoint=True`` uses the matched backprojector instead, which makes the
update the gradient step of 0.5 ||A x - b||^2 (the reference CLI's
--exact-adjoint, src/aprict/scripts/recon_cbfp_landweber.py:486-492).
"""

from __future__ import annotations

import dataclasses
import logging

import numpy as np
import torch

from .. import Volume
from ..cb import flatpanel as fp


@dataclasses.dataclass(frozen=True, kw_only=True)
class _Config:
    """Configuration of the Landweber iterator (landweber_vram.py:54-71)."""

    rayleigh_quotient_num_iterations: int = 10
    acceleration_factor: float = 1
    fast_backproject: bool = True
    soft_from_cylinder_relrad: float | None = 0.95
    bp_soft_from_detedge_relrad: float | None = 0.95
    exact_adjoint: bool = False
    seed: int | None = None


class Landweber_flatpanel:  # noqa: N801
    """An iterable Landweber reconstructor with ordered subsets."""

    Config = _Config

    def __init__(
        self,
        config: _Config,
        volume: Volume,
        projs: fp.ProjectionSet | list[fp.ProjectionSet],
        *,
        proj_zero_masks: torch.Tensor | list[torch.Tensor] | None = None,
        logger: logging.Logger | None = None,
    ) -> None:
        self._logger = logger if logger is not None else logging.getLogger(__name__)
        self._config = config
        self._vol = volume
        self._meas = projs if isinstance(projs, list) else [projs]
        if proj_zero_masks is None:
            self._zm = [None] * len(self._meas)
        elif isinstance(projs, list):
            if not isinstance(proj_zero_masks, list):
                msg = "The input measurements were a list, but only a single mask was provided."
                raise ValueError(msg)
            self._zm = proj_zero_masks
        else:
            if isinstance(proj_zero_masks, list):
                msg = "The input measurements were not a list, but a list of masks was provided."
                raise ValueError(msg)
            self._zm = [proj_zero_masks]
        for p in self._meas:
            if p.data is None:
                msg = "A provided ProjectionSet object has no data."
                raise ValueError(msg)
        sep = 0 if config.bp_soft_from_detedge_relrad is None else (1 - config.bp_soft_from_detedge_relrad)
        if config.exact_adjoint:
            self._config_bp = fp.ConfigBackproject()
        else:
            self._config_bp = fp.ConfigBackproject(
                fast_approx=config.fast_backproject,
                cyl_mask_rad=min(*volume.shape[:2]) / 2 * volume.voxwid,
                apply_summand_multiplier=False,
                soften_det_edges_proportion=sep,
            )
        self._config_fp = fp.ConfigProject()
        self._scratch = [p.zeroed_copy() for p in self._meas]
        self._rq = self.calculate_rayleigh_quotients(config.rayleigh_quotient_num_iterations)
        for p, zm in zip(self._meas, self._zm):
            if zm is not None:
                p.data.mul_(zm)

    def calculate_rayleigh_quotients(self, num_iterations: int) -> list[float]:
        """Largest-eigenvalue estimates of B A, one per ordered subset (power method)."""
        rng = np.random.default_rng(self._config.seed) if self._config.seed is not None else None
        scratch = self._vol.zeroed_copy()
        scale = 1 / float(np.mean(scratch.shape))
        out = []
        for p in self._scratch:
            noise = rng.standard_normal(scratch.shape) if rng is not None else np.random.randn(*scratch.shape)  # noqa: NPY002
            scratch.copy_from(np.abs(noise * scale).astype(np.float32))
            svn = scratch.norm
            rq = 0.0
            for _ in range(num_iterations):
                scratch.multiply(1 / svn)
                p.data.zero_()
                fp.project(self._config_fp, scratch, p, block=True)
                rq = float(torch.linalg.vector_norm(p.data, dtype=torch.float64) ** 2)
                scratch.fill(0)
                fp.backproject(self._config_bp, scratch, p, block=True)
                svn = scratch.norm
            out.append(rq)
        return out

    @property
    def rayleigh_quotients(self) -> list[float]:
        """The per-subset Rayleigh quotients."""
        return list(self._rq)

    def iterate(self) -> None:
        """One pass over the ordered subsets (asynchronous on the current stream)."""
        for meas, scr, rq, zm in zip(self._meas, self._scratch, self._rq, self._zm):
            relax = self._config.acceleration_factor / rq
            if zm is None:
                # r = relax * (b - A x) in one kernel: base = relax*b, mba = -relax
                fp.project_residual(fp.ConfigProject(multiply_before_adding=-relax), self._vol, scr, meas.data * relax)
            else:
                fp.project_residual(fp.ConfigProject(multiply_before_adding=-1), self._vol, scr, meas.data)
                scr.data.mul_(zm).mul_(relax)
            fp.backproject(self._config_bp, self._vol, scr)

    @property
    def volume(self) -> Volume:
        """The volume being reconstructed."""
        return self._vol
