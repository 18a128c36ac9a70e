"""Parity at the benchmark configurations' full sizes against the FP64 oracle.

The other GPU tests use small volumes and detectors; these run the CUDA path at
the sizes the throughput numbers are quoted on and compare with the FP64
restatement (oracle/ab_oracle.c) on the same seeded inputs:

  * c1 -- 128^3 x 1 mm (10 ellipsoids), 180 views on 256^2 x 1 mm pixels,
    SOD 500, SDD 1000: the whole forward projection, the exact (matched)
    backprojection and the fast nearest and bilinear backprojections of all
    180 views;
  * c4 -- 256^3 x 0.5 mm (30 ellipsoids), 360 views on 384^2 x 0.8 mm:
    projection and SIRT-configuration backprojection on a view sample, the
    backprojection of all 360 views (FP32 accumulation over 360 terms per
    voxel; nearest-pixel ties that FP64 cannot settle are counted and left
    out), the dot-product test on the full operator and central finite
    differences on 64 voxels at h = 1e-3;
  * c3 -- 100 clipped quadrics, full 1024^2 views at 0.3 mm, SOD 700, SDD 1200,
    additive in both the reference's parametric form and in length units;
  * c2 -- 4 of the 64 fan-beam slices (512^2 x 0.5 mm, 720 views on 1024 x
    0.4 mm, SOD 600, SDD 1100), Ram-Lak with Hann apodisation, full FBP;
  * c5 -- three scans drawn from the full ranges (edge up to 320, 768^2
    detectors, helical and jittered) through the batched persistent kernels,
    and a 720-view backprojection (the longest accumulation of the batch).

Tolerances are the stated ones: rel L2 <= 1e-5 for projections and
backprojections (adjoints), <= 1e-4 for reconstructions, dot-product
mismatch <= 1e-6. The finite-difference gradient check allows 2e-3 (the loss
differences are FP32 projections of a perturbed volume).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import FBVolume, Volume, geometry, phantoms, ramp_kernels
from aprict_b200.autograd import SiddonProjector
from aprict_b200.batch import ScanBatch
from aprict_b200.cb import flatpanel as fp
from aprict_b200.recon import fan_geometry, fbp_fan_circ_batch
from helpers import rel_l2
from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _corner(shape, voxwid: float) -> np.ndarray:
    return -np.float32(voxwid) * np.array(shape, np.float32) / 2


# ---------------------------------------------------------------- c1
C1 = dict(n=128, voxwid=1.0, views=180, det=256, pix_at_iso=0.5, R=500.0, LmR=500.0, seed=3)


@pytest.fixture(scope="module")
def c1():
    w = C1
    n = w["n"]
    pg = fp.ProjGeom.new_circular_scan(num_source_points=w["views"], R=w["R"], L_minus_R=w["LmR"],
                                       pix_widhei_at_isocenter=(w["pix_at_iso"],) * 2, num_pix_widhei=(w["det"],) * 2)
    x = phantoms.ellipsoid_volume(w["seed"], 10, (n, n, n), w["voxwid"], semi_axes_vox=(5, 40))
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), Volume(x, voxwid=w["voxwid"]), ps, block=True)
    return pg, x, ps


def test_c1_full_projection(c1) -> None:
    pg, x, ps = c1
    want, nseg = O.project_siddon(pg.to_proj_spec_array(), x, voxwid=1.0, corner=_corner(x.shape, 1.0))
    assert nseg > 1e9
    assert rel_l2(ps.data.cpu().numpy(), want) <= 1e-5


@pytest.mark.parametrize("kw", [dict(), dict(fast_approx=True), dict(fast_approx=True, approx_mode_bilinear_interpolate=True)],
                         ids=["exact", "nearest", "bilinear"])
def test_c1_full_backprojection(c1, kw) -> None:
    pg, x, ps = c1
    cfg = fp.ConfigBackproject(**kw)
    out = Volume.zeros(x.shape, voxwid=1.0)
    fp.backproject(cfg, out, ps, block=True)
    p = ps.data.cpu().numpy()
    want = O.backproject(pg.to_proj_spec_array(), p, x.shape, cfg.contents, voxwid=1.0, corner=_corner(x.shape, 1.0))
    assert np.linalg.norm(want) > 0
    assert rel_l2(out.as_numpy(), want) <= 1e-5


# ---------------------------------------------------------------- c4
C4 = dict(n=256, voxwid=0.5, views=360, det=384, pix_at_iso=0.4, R=500.0, LmR=500.0, seed=4)


@pytest.fixture(scope="module")
def c4():
    w = C4
    n = w["n"]
    pg = fp.ProjGeom.new_circular_scan(num_source_points=w["views"], R=w["R"], L_minus_R=w["LmR"],
                                       pix_widhei_at_isocenter=(w["pix_at_iso"],) * 2, num_pix_widhei=(w["det"],) * 2)
    x = phantoms.ellipsoid_volume(w["seed"], 30, (n, n, n), w["voxwid"], semi_axes_vox=(10, 80))
    return pg, x


def _sirt_bp_config(n: int, voxwid: float) -> fp.ConfigBackproject:
    return fp.ConfigBackproject(fast_approx=True, cyl_mask_rad=n / 2 * voxwid, soften_det_edges_proportion=0.05)


def test_c4_projection_and_backprojection_view_sample(c4) -> None:
    pg, x = c4
    sel = [int(i) for i in np.linspace(0, 360, 8, endpoint=False) + 3]
    pgs = pg.sliced(sel)
    ps = fp.ProjectionSet(pgs, data=None)
    v = Volume(x, voxwid=0.5)
    fp.project(fp.ConfigProject(), v, ps, block=True)
    corner = _corner(x.shape, 0.5)
    want, _ = O.project_siddon(pgs.to_proj_spec_array(), x, voxwid=0.5, corner=corner)
    assert rel_l2(ps.data.cpu().numpy(), want) <= 1e-5
    for cfg in (_sirt_bp_config(256, 0.5), fp.ConfigBackproject(fast_approx=True, approx_mode_bilinear_interpolate=True)):
        out = Volume.zeros(x.shape, voxwid=0.5)
        fp.backproject(cfg, out, ps, block=True)
        want_b = O.backproject(pgs.to_proj_spec_array(), ps.data.cpu().numpy(), x.shape, cfg.contents, voxwid=0.5,
                               corner=corner)
        assert rel_l2(out.as_numpy(), want_b) <= 1e-5


@pytest.mark.parametrize("theta0", [0.0, 0.0123])
def test_c4_backprojection_all_views(c4, theta0: float) -> None:
    # 360 views accumulate per voxel in FP32: the whole sum against the FP64
    # oracle, with random data (every nearest-pixel choice shows). At theta0 = 0
    # the views at 45, 135, 225 and 315 degrees see the voxels of the two
    # diagonal planes exactly on the boundary of the detector's centre column
    # (an even detector width): those choices are ties that FP64 cannot settle
    # (both evaluations are within rounding of the half-integer), so voxels
    # holding such a tie are left out of the comparison and counted.
    pg0, x = c4
    pg = pg0 if theta0 == 0.0 else fp.ProjGeom.new_circular_scan(
        num_source_points=360, R=500.0, L_minus_R=500.0, pix_widhei_at_isocenter=(0.4, 0.4),
        num_pix_widhei=(384, 384), theta_start=theta0)
    rng = np.random.default_rng(8)
    data = (rng.random((360, 384, 384), dtype=np.float32) + 0.5)
    ps = fp.ProjectionSet(pg, data=data)
    cfg = _sirt_bp_config(256, 0.5)
    out = Volume.zeros(x.shape, voxwid=0.5)
    fp.backproject(cfg, out, ps, block=True)
    specs, corner = pg.to_proj_spec_array(), _corner(x.shape, 0.5)
    want = O.backproject(specs, data, x.shape, cfg.contents, voxwid=0.5, corner=corner)
    ties = O.bp_nearest_ties(specs, x.shape, cfg.contents, voxwid=0.5, corner=corner) > 0
    assert ties.mean() <= (0.01 if theta0 == 0.0 else 1e-5)
    keep = ~ties
    assert rel_l2(out.as_numpy()[keep], want[keep]) <= 1e-5


def test_c4_dot_product_full_operator(c4) -> None:
    pg, x = c4
    proj = SiddonProjector(pg, x.shape, voxwid=0.5)
    g = torch.Generator("cuda").manual_seed(11)
    xr = torch.rand(x.shape, device="cuda", generator=g)
    y = torch.rand(proj.data_shape, device="cuda", generator=g)
    lhs = float((proj.forward_raw(xr).double() * y.double()).sum())
    rhs = float((xr.double() * proj.adjoint_raw(y).double()).sum())
    assert abs(lhs - rhs) / abs(lhs) <= 1e-6


def test_c4_central_finite_differences(c4) -> None:
    pg, xt = c4
    proj = SiddonProjector(pg, xt.shape, voxwid=0.5)
    xt_d = torch.from_numpy(xt).cuda()
    g = torch.Generator("cuda").manual_seed(12)
    b = proj.forward_raw(xt_d) + 0.01 * torch.randn(proj.data_shape, device="cuda", generator=g)
    x0 = 0.8 * xt_d
    x = x0.clone().requires_grad_(True)
    (0.5 * ((proj(x) - b).double() ** 2).sum()).backward()
    grad = x.grad.double()

    def loss(v: torch.Tensor) -> float:
        return float(0.5 * ((proj.forward_raw(v) - b).double() ** 2).sum())

    rng = np.random.default_rng(13)
    h = 1e-3
    fd, an = [], []
    for _ in range(64):
        i = tuple(int(rng.integers(64, 192)) for _ in range(3))
        xp, xm = x0.clone(), x0.clone()
        xp[i] += h
        xm[i] -= h
        fd.append((loss(xp) - loss(xm)) / (2 * h))
        an.append(float(grad[i]))
    fd, an = np.array(fd), np.array(an)
    assert np.linalg.norm(an) > 0
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) <= 2e-3


# ---------------------------------------------------------------- c3
@pytest.mark.parametrize("kw", [dict(overlap_addition=True), dict(overlap_addition=True, additive_line_integral=True)],
                         ids=["parametric", "length"])
def test_c3_quadric_full_views(kw) -> None:
    R, L = 700.0, 1200.0  # noqa: N806
    pg = fp.ProjGeom.new_circular_scan(num_source_points=720, R=R, L_minus_R=L - R,
                                       pix_widhei_at_isocenter=(0.3 * R / L,) * 2, num_pix_widhei=(1024, 1024))
    shapes = phantoms.random_quadric_phantom(11, n_ellipsoids=60, n_cylinders=40, radius=100.0)
    pgs = pg.sliced([5, 187, 433])
    ps = fp.ProjectionSet(pgs, data=None)
    cfg = fp.ConfigProject(**kw)
    fp.project(cfg, FBVolume(shapes), ps, block=True)
    mode = 2 if kw.get("additive_line_integral") else 1
    want = O.project_forbild(pgs.to_proj_spec_array(), shapes, mode=mode)
    assert np.count_nonzero(want) > 1e5
    assert rel_l2(ps.data.cpu().numpy(), want) <= 1e-5


# ---------------------------------------------------------------- c2
def test_c2_fan_fbp_four_slices() -> None:
    from scipy.signal import fftconvolve

    n, views, nu, R, LmR = 512, 720, 1024, 600.0, 500.0  # noqa: N806
    L = R + LmR  # noqa: N806
    pg = fp.ProjGeom.new_circular_scan(num_source_points=views, R=R, L_minus_R=LmR,
                                       pix_widhei_at_isocenter=(0.4 * R / L,) * 2, num_pix_widhei=(nu, 1))
    projs, outs = [], []
    for k in range(4):
        x = phantoms.ellipsoid_volume(70 + k, 20, (n, n, 1), 0.5, semi_axes_vox=(8, 160))
        ps = fp.ProjectionSet(pg, data=None)
        fp.project(fp.ConfigProject(), Volume(x, voxwid=0.5), ps, block=True)
        projs.append(ps)
        outs.append(Volume.zeros((n, n, 1), voxwid=0.5))
    fbp_fan_circ_batch(projs, outs, apodization="hann")
    Rg, Lg, pixwid, nu_, _ = fan_geometry(pg)  # noqa: N806
    u = pixwid / Lg * (np.arange(nu) - (nu - 1) / 2)
    wgt = 1.0 / np.sqrt(1 + u**2)
    taps = ramp_kernels.apodize_hann(ramp_kernels.ramp_kernel_ramlak(2 * nu - 1, pixwid / Lg))
    cfg = fp.ConfigBackproject(fast_approx=True, cyl_mask_rad=Rg * np.sin(np.arctan(pixwid * nu / 2 / Lg)),
                               Z_on_val_factor_power=-2, Z_on_val_factor_val=Rg, approx_mode_direct_raycast=True)
    for ps, out in zip(projs, outs):
        p = ps.data.cpu().numpy().astype(np.float64)[:, :, 0] * wgt
        filt = fftconvolve(p, taps[None, :], mode="full", axes=1)[:, nu - 1 : 2 * nu - 1]
        filt = (filt / (4 * np.pi * Rg * views))[:, :, None]
        want = O.backproject(pg.to_proj_spec_array(), filt, (n, n, 1), cfg.contents, voxwid=0.5,
                             corner=_corner((n, n, 1), 0.5))
        assert np.linalg.norm(want) > 0
        assert rel_l2(out.as_numpy(), want) <= 1e-4


# ---------------------------------------------------------------- c5
def _c5_scans():
    rng = np.random.default_rng(5)
    params = geometry.uneven_scans(rng, 48, edge=(64, 320), views=(90, 720), det=(128, 768), voxwid=0.5)
    # the largest volume, the largest detector and the first helical scan of the batch
    big = max(range(48), key=lambda i: params[i]["n"])
    wide = max(range(48), key=lambda i: params[i]["det"])
    hel = next(i for i in range(48) if params[i]["helical"] and i not in (big, wide))
    picks = [big, wide, hel]
    geos = {}
    for i, s in enumerate(params):  # the same draws as the batch workload's scan list
        pg = geometry.scan_geometry(rng, s)
        if i in picks:
            geos[i] = pg
    return [(params[i], geos[i]) for i in picks]


def test_c5_batched_scans_at_full_ranges() -> None:
    scans = _c5_scans()
    assert max(s["n"] for s, _ in scans) >= 250 and max(s["det"] for s, _ in scans) >= 700
    vols, sub_pgs, xs = [], [], []
    for k, (s, pg) in enumerate(scans):
        n = s["n"]
        x = phantoms.ellipsoid_volume(500 + k, 10, (n, n, n), 0.5, semi_axes_vox=(max(2.0, n / 32), n / 6))
        xs.append(x)
        vols.append(Volume(x, voxwid=0.5))
        m = pg.num_projs
        sub_pgs.append(pg.sliced([int(i) for i in np.linspace(0, m, 4, endpoint=False)]))
    projs = [fp.ProjectionSet(pg, data=None) for pg in sub_pgs]
    ScanBatch(vols, projs).project(block=True)
    cfg = fp.ConfigBackproject(fast_approx=True, soften_det_edges_proportion=0.05)
    outs = [v.zeroed_copy() for v in vols]
    ScanBatch(outs, projs).backproject(cfg, block=True)
    for x, pg, p, o in zip(xs, sub_pgs, projs, outs):
        corner = _corner(x.shape, 0.5)
        want, _ = O.project_siddon(pg.to_proj_spec_array(), x, voxwid=0.5, corner=corner)
        assert rel_l2(p.data.cpu().numpy(), want) <= 1e-5
        want_b = O.backproject(pg.to_proj_spec_array(), p.data.cpu().numpy(), x.shape, cfg.contents, voxwid=0.5,
                               corner=corner)
        assert np.linalg.norm(want_b) > 0
        assert rel_l2(o.as_numpy(), want_b) <= 1e-5


def test_c5_backprojection_720_views() -> None:
    # the longest accumulation of the batch: 720 views into each voxel, batched kernel
    rng = np.random.default_rng(6)
    s = dict(n=128, views=720, det=384, helical=True, pitch=1.0, pix_at_iso=1.5 * 128 * 0.5 / 384, voxwid=0.5,
             R=500.0, L_minus_R=500.0, theta0=0.4)
    pg = geometry.scan_geometry(rng, s)
    data = rng.random((720, 384, 384), dtype=np.float32) + 0.5
    cfg = fp.ConfigBackproject(fast_approx=True, soften_det_edges_proportion=0.05)
    out = Volume.zeros((128, 128, 128), voxwid=0.5)
    ScanBatch([out], [fp.ProjectionSet(pg, data=data)]).backproject(cfg, block=True)
    want = O.backproject(pg.to_proj_spec_array(), data, (128, 128, 128), cfg.contents, voxwid=0.5,
                         corner=_corner((128, 128, 128), 0.5))
    assert np.linalg.norm(want) > 0
    assert rel_l2(out.as_numpy(), want) <= 1e-5
