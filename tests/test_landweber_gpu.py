"""Landweber_flatpanel on the GPU vs an FP64 restatement of the reference's iterator.

The restatement follows src/aprict/iterators/landweber_vram.py step by step:
  * Rayleigh quotients (:127-209): per ordered subset a start volume
    |randn(shape) / mean(shape)| (float32) drawn from numpy's global generator,
    then num_iterations power steps v <- v / |v|; p = A v; rho = |p|^2;
    v = B p; |v| recomputed;
  * the update (:221-260): for each subset r = b - A x, r *= zero mask,
    x += (accel / rho) B r;
with A the FP64 Siddon oracle and B the FP64 fast backprojection (cylinder mask
and 5 % detector-edge taper, :104-109). Both sides draw their start volumes
after the same numpy global seed, as a reference user seeding numpy would.

Gates: Rayleigh quotients rel 1e-5 (a projection-level quantity); the volume
after three passes over the subsets rel L2 1e-4 (reconstruction tolerance).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import Volume, phantoms
from aprict_b200.cb import flatpanel as fp
from aprict_b200.iterators import Landweber_flatpanel
from helpers import circular, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPE = (40, 36, 30)


class OracleLandweber:
    """FP64 restatement of Landweber_flatpanel (ordered subsets, power-method step sizes)."""

    def __init__(self, pgs, bs, masks, cfg_contents, *, accel: float, num_iterations: int) -> None:
        self.specs = [pg.to_proj_spec_array() for pg in pgs]
        self.corner = -np.array(SHAPE, np.float32) / 2
        self.cfg = cfg_contents
        self.accel = accel
        self.x = np.zeros(SHAPE)
        scale = 1 / float(np.mean(SHAPE))
        self.rq = []
        for k in range(len(self.specs)):
            v = np.abs(np.random.randn(*SHAPE) * scale).astype(np.float32).astype(np.float64)  # noqa: NPY002
            svn = np.linalg.norm(v)
            rq = 0.0
            for _ in range(num_iterations):
                v = v / svn
                p = self.A(k, v)
                rq = float(np.sum(p * p))
                v = self.B(k, p)
                svn = np.linalg.norm(v)
            self.rq.append(rq)
        self.b = [b.astype(np.float64) * (1 if m is None else m) for b, m in zip(bs, masks)]
        self.masks = masks

    def A(self, k: int, x: np.ndarray) -> np.ndarray:  # noqa: N802
        return O.project_siddon(self.specs[k], x, voxwid=1.0, corner=self.corner)[0]

    def B(self, k: int, p: np.ndarray) -> np.ndarray:  # noqa: N802
        return O.backproject(self.specs[k], p, SHAPE, self.cfg, voxwid=1.0, corner=self.corner)

    def iterate(self) -> None:
        for k in range(len(self.specs)):
            r = self.b[k] - self.A(k, self.x)
            if self.masks[k] is not None:
                r = r * self.masks[k]
            self.x = self.x + (self.accel / self.rq[k]) * self.B(k, r)


def _subsets(n_subsets: int):
    pg = circular(36, 110, 110, 0.537, 52, 44)
    xt = phantoms.ellipsoid_volume(41, 6, SHAPE, 1.0, semi_axes_vox=(3, 12))
    v = Volume(xt, voxwid=1.0)
    pgs, bs = [], []
    for k in range(n_subsets):
        sub = pg.sliced(list(range(k, 36, n_subsets)))  # interleaved ordered subsets
        ps = fp.ProjectionSet(sub, data=None)
        fp.project(fp.ConfigProject(), v, ps, block=True)
        pgs.append(sub)
        bs.append(ps.data.cpu().numpy())
    return pgs, bs


@pytest.mark.parametrize("n_subsets,masked", [(1, False), (3, True)])
def test_landweber_matches_fp64_restatement(n_subsets: int, masked: bool) -> None:
    pgs, bs = _subsets(n_subsets)
    rng = np.random.default_rng(17)
    masks = [(rng.random(b.shape) > 0.05).astype(np.float32) if masked else None for b in bs]
    cfg = Landweber_flatpanel.Config(acceleration_factor=1.5)
    np.random.seed(1234)  # noqa: NPY002  the start volumes come from numpy's global generator
    x = Volume.zeros(SHAPE, voxwid=1.0)
    projs = [fp.ProjectionSet(pg, data=b.copy()) for pg, b in zip(pgs, bs)]
    zm = None
    if masked:
        zm = [torch.from_numpy(m).cuda() for m in masks]
    lw = Landweber_flatpanel(cfg, x, projs if n_subsets > 1 else projs[0],
                             proj_zero_masks=zm if n_subsets > 1 else (zm[0] if zm else None))
    np.random.seed(1234)  # noqa: NPY002
    ora = OracleLandweber(pgs, bs, masks, lw._config_bp.contents, accel=1.5,  # noqa: SLF001
                          num_iterations=cfg.rayleigh_quotient_num_iterations)
    for got, want in zip(lw.rayleigh_quotients, ora.rq):
        assert abs(got - want) / want <= 1e-5
    for _ in range(3):
        lw.iterate()
        ora.iterate()
    torch.cuda.synchronize()
    assert np.linalg.norm(ora.x) > 0
    assert rel_l2(x.as_numpy(), ora.x) <= 1e-4


def test_landweber_exact_adjoint_is_gradient_step() -> None:
    # --exact-adjoint: the matched backprojector makes each update the gradient
    # step of 0.5 |A x - b|^2, with the oracle's transpose of A
    pgs, bs = _subsets(1)
    cfg = Landweber_flatpanel.Config(exact_adjoint=True, rayleigh_quotient_num_iterations=6)
    x = Volume.zeros(SHAPE, voxwid=1.0)
    np.random.seed(7)  # noqa: NPY002
    lw = Landweber_flatpanel(cfg, x, fp.ProjectionSet(pgs[0], data=bs[0].copy()))
    specs = pgs[0].to_proj_spec_array()
    corner = -np.array(SHAPE, np.float32) / 2
    xo = np.zeros(SHAPE)
    for _ in range(2):
        lw.iterate()
        r = bs[0].astype(np.float64) - O.project_siddon(specs, xo, voxwid=1.0, corner=corner)[0]
        xo = xo + O.backproject_transpose(specs, r, SHAPE, voxwid=1.0, corner=corner) / lw.rayleigh_quotients[0]
    torch.cuda.synchronize()
    assert rel_l2(x.as_numpy(), xo) <= 1e-4
