"""GBC on the GPU vs the FP64 oracle (pinned to the reference in test_gbc.py).

* Preset-7 backprojection into the volume and the weight-sum volume
  (nearest and bilinear, supersampling, summand multiplier, C and F order):
  rel L2 <= 1e-5 against the oracle.
* The expected weight-sum integral: rel <= 1e-5.
* The cone-beam volume filter (cuFFT + the fused spectral kernel), with and
  without the low-resolution correction, cone angles 0 < a < pi, 0 and pi:
  rel L2 <= 1e-5; the upsampling kernel against scipy.ndimage.map_coordinates.
* Volume ops: soft-zero division and the xy-grid product.
* The GBC driver on a small cylindrical scan against the oracle driver:
  rel L2 <= 1e-4.
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.ndimage
import torch

from aprict_b200 import Volume, _lib, gbc, phantoms
from aprict_b200.cb import flatpanel as fp
from aprict_b200.recon import fan_geometry, gbc_cone_cyl
from helpers import rel_l2
from oracle import gbc as G

pytestmark = pytest.mark.gpu

SOFT = (0.22, 0.05, 0.45, 0.05)


def _scan(m: int = 20, R: float = 60.0, LmR: float = 60.0, pix: float = 1.3, nu: int = 30, nv: int = 22,  # noqa: N803
          h: float = 12.0) -> fp.ProjGeom:
    ts = 0.3 + np.arange(m) * (np.sqrt(5) - 1) * np.pi
    zs = np.linspace(-h / 2, h / 2, m + 2)[1:-1]
    src = np.stack([R * np.cos(ts), R * np.sin(ts), zs], 1)
    det = np.stack([-LmR * np.cos(ts), -LmR * np.sin(ts), zs], 1)
    u = pix * np.stack([-np.sin(ts), np.cos(ts), 0 * ts], 1)
    v = np.broadcast_to(pix * np.array([0.0, 0.0, -1.0]), (m, 3)).copy()
    return fp.ProjGeom(source_pos=src, det_pos=det, det_uvec=u, det_vvec=v, nu=nu, nv=nv)


def _cfg(linear: bool, ss: int = 1, mult: bool = False) -> fp.ConfigBackproject:
    return fp.ConfigBackproject(fast_approx=True, backproj_weighting_preset=7, Z_on_val_factor_val=60.0,
                                approx_mode_direct_raycast=True, approx_mode_bilinear_interpolate=linear,
                                apply_summand_multiplier=mult, ssx=ss, ssy=ss, ssz=ss, soft_vartheta_v=SOFT[0],
                                soft_vartheta_v_softspan=SOFT[1], soft_vartheta_h=SOFT[2],
                                soft_vartheta_h_softspan=SOFT[3])


@pytest.mark.parametrize(("linear", "ss", "order", "mult"), [(False, 1, "C", False), (True, 1, "F", True),
                                                             (False, 2, "F", True), (True, 2, "C", False)])
def test_backprojection_matches_oracle(linear: bool, ss: int, order: str, mult: bool) -> None:
    pg = _scan()
    rng = np.random.default_rng(4)
    projs = rng.random((pg.num_projs, 30, 22)).astype(np.float32)
    shape, vw = (11, 13, 9), 1.7
    v = Volume.zeros(shape, voxwid=vw, pos_c=(0.3, -0.2, 0.5), order=order)
    ws = Volume.zeros(shape, voxwid=vw, pos_c=(0.3, -0.2, 0.5), order=order)
    v.fill(0.25)
    m = rng.uniform(0.5, 1.5, shape).astype(np.float32) if mult else None
    mv = Volume(m, voxwid=vw, pos_c=(0.3, -0.2, 0.5), order=order) if mult else None
    fp.backproject(_cfg(linear, ss, mult), v, fp.ProjectionSet(pg, data=projs), secondary_volume=ws,
                   summand_multiplier=mv, block=True)
    w1, w2 = G.backproject_gbc(pg.to_proj_spec_array(), projs, shape, vw, v.corner, R=60.0, soft=SOFT, linear=linear,
                               ss=(ss, ss, ss), mult=m)
    assert np.linalg.norm(w1) > 0 and np.linalg.norm(w2) > 0
    assert rel_l2(v.as_numpy() - 0.25, w1) <= 1e-5
    assert rel_l2(ws.as_numpy(), w2) <= 1e-5


def test_preset7_needs_secondary_volume() -> None:
    pg = _scan(m=2)
    v = Volume.zeros((4, 4, 4), voxwid=1.0)
    with pytest.raises(ValueError):
        fp.backproject(_cfg(False), v, fp.ProjectionSet(pg, data=np.ones((2, 30, 22), np.float32)))


def test_weight_integral_matches_oracle() -> None:
    cfg = _cfg(False)
    r = np.linspace(0.0, 0.4, 9)
    got = gbc.backproj_gbc_weight_integ_GPU(r, cfg, 120, 90)
    want = G.weight_integral(r.astype(np.float32), SOFT, 120, 90)
    assert np.all(want > 0)
    np.testing.assert_allclose(got, want, rtol=1e-5)


@pytest.mark.parametrize(("r", "nz", "na", "soft"), [
    (np.array([0.3]), 2, 1, SOFT),                      # smallest sampling
    (np.array([0.0, 0.5, 0.9]), 3, 7, SOFT),
    (np.linspace(0.0, 0.3, 5), 400, 300, (2.0, 0.1, 1.7, 0.3)),  # windows past pi/2: nothing cut
    (np.linspace(0.0, 0.3, 4), 300, 257, (0.1, 0.2, 0.45, 0.05)),  # soft span wider than the window
    (np.linspace(0.0, 0.3, 3), 300, 200, (1.7, 0.3, 0.45, 0.05)),  # past pi/2: heights below 0, soft band in use
])
def test_weight_integral_edges(r: np.ndarray, nz: int, na: int, soft: tuple) -> None:
    cfg = fp.ConfigBackproject(fast_approx=True, backproj_weighting_preset=7, Z_on_val_factor_val=60.0,
                               approx_mode_direct_raycast=True, soft_vartheta_v=soft[0],
                               soft_vartheta_v_softspan=soft[1], soft_vartheta_h=soft[2],
                               soft_vartheta_h_softspan=soft[3])
    got = gbc.backproj_gbc_weight_integ_GPU(r, cfg, nz, na)
    want = G.weight_integral(r.astype(np.float32), soft, nz, na)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6 * max(1.0, float(np.abs(want).max())))


@pytest.mark.parametrize(("cone", "soft"), [(0.5, 0.05), (0.0, 0.0), (np.pi, 0.0), (1.2, 0.2)])
def test_conebeam_filter_matches_oracle(cone: float, soft: float) -> None:
    rng = np.random.default_rng(int(cone * 10))
    a = rng.standard_normal((20, 18, 24)).astype(np.float32)
    got = gbc.ramp_filter_conebeam(a, 0.7, cone, soft)
    want = G.ramp_filter_conebeam(a, 0.7, cone, soft)
    assert isinstance(got, np.ndarray) and got.shape == a.shape
    assert rel_l2(got, want) <= 1e-5
    # device input, low-resolution correction, extra multiplier
    low = rng.standard_normal((10, 9, 12)).astype(np.float32)
    got2 = gbc.ramp_filter_conebeam(torch.from_numpy(a).cuda(), 0.7, cone, soft, lowres_correction_array=low,
                                    extra_multiplier=2.0)
    want2 = G.ramp_filter_conebeam(a, 0.7, cone, soft, lowres=low, extra_multiplier=2.0)
    assert rel_l2(got2.cpu().numpy(), want2) <= 1e-5


def test_upsampling_kernel_is_map_coordinates() -> None:
    rng = np.random.default_rng(8)
    shape, d = (15, 12, 21), 3
    low = rng.standard_normal((5, 4, 7)).astype(np.float32)
    out = torch.zeros(shape, device="cuda")
    lo = torch.from_numpy(low).cuda()
    _lib.check(_lib.lib().aprict_b200_add_upsampled(out.data_ptr(), *shape, lo.data_ptr(), *low.shape, d,
                                                    torch.cuda.current_stream().cuda_stream), "add_upsampled")
    coords = np.meshgrid(*[np.arange(n) / d - 0.5 + 1 / d / 2 for n in shape], indexing="ij")
    want = scipy.ndimage.map_coordinates(low.astype(np.float64), coords, order=1, mode="nearest")
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("order", ["C", "F"])
def test_volume_ops(order: str) -> None:
    rng = np.random.default_rng(9)
    a = rng.standard_normal((6, 7, 5)).astype(np.float32)
    w = rng.uniform(-1e-5, 2.0, (6, 7, 5)).astype(np.float32)
    g = rng.uniform(0.5, 2.0, (6, 7)).astype(np.float32)
    va, vw_ = Volume(a, voxwid=1.0, order=order), Volume(w, voxwid=1.0, order=order)
    va.divide_softzero(vw_, eps=1e-3)
    want = a * (1 / (w + np.float32(1e-3) * np.exp(-w / np.float32(1e-3))))
    np.testing.assert_allclose(va.as_numpy(), want, rtol=2e-6)
    vb = Volume(a, voxwid=1.0, order=order)
    vb.multiply_by_xygrid(g)
    np.testing.assert_array_equal(vb.as_numpy(), a * g[:, :, None])


def test_gbc_reconstruction_matches_oracle() -> None:
    n_vox, vw = 8, 2.0
    pg = _scan(m=36, R=60.0, LmR=60.0, pix=1.6, nu=40, nv=26, h=24.0)
    x = phantoms.ellipsoid_volume(3, 4, (n_vox, n_vox, n_vox), vw, semi_axes_vox=(1.5, 3))
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), Volume(x, voxwid=vw), ps, block=True)
    kw = dict(n=3, f1=1.2, f2=4.0, eps=1e-6, softspan_v=0.05, softspan_h=0.05)
    got = gbc_cone_cyl(ps, (n_vox,) * 3, vw, interpolate_measurements=True, num_z_samps=150, num_ang_samps=150,
                       **kw).as_numpy()
    R, L, pixwid, nu, nv = fan_geometry(pg)  # noqa: N806
    want = G.gbc_cone_cyl(pg.to_proj_spec_array(), ps.data.cpu().numpy(), (n_vox,) * 3, vw, (0.0, 0.0, 0.0), R=R,
                          L=L, pixwid=pixwid, nu=nu, nv=nv, zs=pg.source_pos[:, 2], linear=True, num_z=150,
                          num_ang=150, **kw)
    assert got.shape == want.shape == (n_vox,) * 3
    assert np.linalg.norm(want) > 0
    assert rel_l2(got, want) <= 1e-4
