"""Fan-beam FBP (recon.fbp_fan_circ) vs an FP64 pipeline built from the oracle pieces.

The oracle pipeline restates the reference's fan-beam path
(src/aprict/scripts/recon_cbfp_cyl_fbp.py:368-701, 1108-1121, 1238): cosine
weight, Ram-Lak convolution at pitch pixwid/L (FP64 numpy), direct-raycast
backprojection with (Z/R)^-2 inside the support cylinder (FP64 oracle), scale
1/(4 pi R M). Gate: rel L2 <= 1e-4 (reconstruction tolerance).
"""

from __future__ import annotations

import numpy as np
import pytest

from aprict_b200 import Volume, phantoms, ramp_kernels
from aprict_b200.cb import flatpanel as fp
from aprict_b200.recon import fan_geometry, fbp_fan_circ
from helpers import circular, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _fan_problem(n: int = 96, views: int = 180, nu: int = 192, apod: str | None = None):
    pg = circular(views, 120.0, 100.0, 0.5123, nu, 1, theta0=0.0)
    x = phantoms.ellipsoid_volume(31, 8, (n, n, 1), 0.5, semi_axes_vox=(4, 30))
    v = Volume(x, voxwid=0.5)
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), v, ps, block=True)
    return pg, x, ps


@pytest.mark.parametrize("apod", [None, "hann"])
def test_fbp_matches_fp64_pipeline(apod: str | None) -> None:
    n = 96
    pg, _, ps = _fan_problem(n=n, apod=apod)
    out = Volume.zeros((n, n, 1), voxwid=0.5)
    fbp_fan_circ(ps, out, apodization=apod)
    got = out.as_numpy()

    R, L, pixwid, nu, nv = fan_geometry(pg)  # noqa: N806
    m = pg.num_projs
    p = ps.data.cpu().numpy().astype(np.float64)
    u = pixwid / L * (np.arange(nu) - (nu - 1) / 2)
    w = 1.0 / np.sqrt(1 + u**2)
    taps = ramp_kernels.ramp_kernel_ramlak(2 * nu - 1, pixwid / L)
    if apod == "hann":
        taps = ramp_kernels.apodize_hann(taps)
    filt = np.empty_like(p)
    for i in range(m):
        filt[i, :, 0] = np.convolve(p[i, :, 0] * w, taps, mode="full")[nu - 1 : 2 * nu - 1]
    filt /= 4 * np.pi * R * m
    cfg = fp.ConfigBackproject(
        fast_approx=True, cyl_mask_rad=R * np.sin(np.arctan(pixwid * nu / 2 / L)), Z_on_val_factor_power=-2,
        Z_on_val_factor_val=R, approx_mode_direct_raycast=True,
    )
    want = O.backproject(pg.to_proj_spec_array(), filt, (n, n, 1), cfg.contents, voxwid=0.5, corner=-np.array((n, n, 1), np.float32) * 0.25)
    assert np.linalg.norm(want) > 0
    assert rel_l2(got, want) <= 1e-4


def test_fbp_reconstructs_phantom() -> None:
    n = 128
    pg, x, ps = _fan_problem(n=n, views=360, nu=256)
    out = Volume.zeros((n, n, 1), voxwid=0.5)
    fbp_fan_circ(ps, out, interpolate=True)
    rec = out.as_numpy()
    inside = np.hypot(*np.meshgrid(np.arange(n) - (n - 1) / 2, np.arange(n) - (n - 1) / 2, indexing="ij"))[..., None] < 0.45 * n
    err = np.linalg.norm((rec - x)[inside]) / np.linalg.norm(x[inside])
    assert err < 0.35, err  # discretised FBP of a piecewise-constant phantom: edges dominate the error
    assert abs(rec[inside].mean() - x[inside].mean()) < 0.05 * x[inside].mean()


def test_batched_slices_equal_single_slice_fbp() -> None:
    from aprict_b200.recon import fbp_fan_circ_batch

    n = 64
    pgs = circular(120, 120.0, 100.0, 0.5123, 128, 1, theta0=0.0)
    projs, singles = [], []
    for k in range(5):
        x = phantoms.ellipsoid_volume(40 + k, 6, (n, n, 1), 0.5, semi_axes_vox=(3, 20))
        ps = fp.ProjectionSet(pgs, data=None)
        fp.project(fp.ConfigProject(), Volume(x, voxwid=0.5), ps, block=True)
        projs.append(ps)
        one = Volume.zeros((n, n, 1), voxwid=0.5)
        fbp_fan_circ(ps, one, apodization="hann")
        singles.append(one.as_numpy())
    outs = [Volume.zeros((n, n, 1), voxwid=0.5) for _ in range(5)]
    fbp_fan_circ_batch(projs, outs, apodization="hann")
    for o, w in zip(outs, singles):
        assert np.linalg.norm(w) > 0
        assert rel_l2(o.as_numpy(), w) <= 1e-6
