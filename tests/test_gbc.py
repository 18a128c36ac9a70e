"""GBC pieces on the CPU: the FP64 oracle pinned against the reference.

* The oracle's GBC weight against the reference's own _GBC_weightfun<float>
  (src/aprict/data/cusrc/CB_backproject.cu:736-787, compiled for the CPU).
* The oracle's GBC backprojection (volume and weight sums) against the
  reference's backproject_CB_voltex_GBC_cyl<float,float> (:1030-1105),
  launched per 10 views as flatpanel.backproject does for preset 7.
* The k-factor of the softened Colsher window (gbc/filters.py:59-147): 2 pi
  outside the band, continuous at its edges, symmetric about pi/2, in
  (0, 2 pi].
* The oracle's low-resolution upsampling against scipy.ndimage.map_coordinates
  (order 1, mode "nearest"), the published definition behind the reference's
  cupyx call (gbc/filters.py:403-455).
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.ndimage

from aprict_b200.cb import flatpanel as fp
from helpers import rel_l2
from oracle import gbc as G
from oracle import oracle as O

SOFT = (0.22, 0.05, 0.45, 0.05)


def _gbc_scan(m: int = 14, R: float = 60.0, LmR: float = 60.0, pix: float = 1.3, nu: int = 30, nv: int = 22):  # noqa: N803
    ts = 0.3 + np.arange(m) * (np.sqrt(5) - 1) * np.pi
    zs = np.linspace(-6, 6, m)
    src = np.stack([R * np.cos(ts), R * np.sin(ts), zs], 1)
    det = np.stack([-LmR * np.cos(ts), -LmR * np.sin(ts), zs], 1)
    u = pix * np.stack([-np.sin(ts), np.cos(ts), 0 * ts], 1)
    v = np.broadcast_to(pix * np.array([0.0, 0.0, -1.0]), (m, 3)).copy()
    return fp.ProjGeom(source_pos=src, det_pos=det, det_uvec=u, det_vvec=v, nu=nu, nv=nv)


@pytest.mark.skipif(not O.have_ref(), reason="reference oracle not built")
def test_weight_matches_reference() -> None:
    rng = np.random.default_rng(2)
    n, R = 4000, 80.0  # noqa: N806
    t = rng.uniform(0, 2 * np.pi, n)
    src = np.stack([R * np.cos(t), R * np.sin(t), rng.uniform(-20, 20, n)], 1)
    vox = rng.uniform(-30, 30, (n, 3))
    want = O.ref_gbc_weight(R, vox, src, np.array(SOFT))
    got = G.gbc_weight(R, vox.astype(np.float32).astype(np.float64), src.astype(np.float32).astype(np.float64), SOFT)
    assert np.count_nonzero(want) > n // 3 and np.count_nonzero(want != 1) > n // 3
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=2e-5)


@pytest.mark.skipif(not O.have_ref(), reason="reference oracle not built")
@pytest.mark.parametrize("linear", [False, True])
def test_backprojection_matches_reference(linear: bool) -> None:
    pg = _gbc_scan()
    rng = np.random.default_rng(3)
    projs = rng.random((pg.num_projs, 30, 22)).astype(np.float32)
    shape, vw = (10, 12, 9), 1.7
    corner = -np.array(shape, np.float32) * np.float32(vw / 2) + np.float32(0.3)
    cfg = fp.ConfigBackproject(fast_approx=True, backproj_weighting_preset=7, Z_on_val_factor_val=60.0,
                               approx_mode_direct_raycast=True, approx_mode_bilinear_interpolate=linear,
                               soft_vartheta_v=SOFT[0], soft_vartheta_v_softspan=SOFT[1], soft_vartheta_h=SOFT[2],
                               soft_vartheta_h_softspan=SOFT[3]).contents
    v1, v2 = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
    O.ref_backproject_gbc(pg.to_proj_spec_array(), projs, v1, v2, cfg, voxwid=vw, corner=corner)
    w1, w2 = G.backproject_gbc(pg.to_proj_spec_array(), projs, shape, vw, corner, R=60.0, soft=SOFT, linear=linear)
    assert np.linalg.norm(w2) > 0 and np.linalg.norm(w1) > 0
    assert rel_l2(v2, w2) <= 2e-6
    # nearest: the reference rounds FP32 detector coordinates, a few voxel-views pick the neighbour
    assert rel_l2(v1, w1) <= (1e-5 if linear else 2e-3)


def test_kfactor_properties() -> None:
    cone, soft = 0.6, 0.05
    h = cone / 2 - soft
    th = np.linspace(0, np.pi, 2001)
    k = G.conebeam_kfactor(th, cone, soft)
    assert np.all(k[th <= h] == 2 * np.pi) and np.all(k[th >= np.pi - h] == 2 * np.pi)
    assert np.all(k > 0) and np.all(k <= 2 * np.pi + 1e-9)
    np.testing.assert_allclose(k, k[::-1], rtol=1e-9)
    edge = G.conebeam_kfactor(np.array([h + 1e-7, np.pi - h - 1e-7]), cone, soft)
    np.testing.assert_allclose(edge, 2 * np.pi, rtol=1e-5)
    assert np.all(G.conebeam_kfactor(th, np.pi, 0.0) == 2 * np.pi)


@pytest.mark.parametrize(("shape", "d"), [((9, 12, 6), 3), ((10, 5, 15), 5), ((7, 7, 7), 1)])
def test_upsampling_is_map_coordinates(shape: tuple[int, int, int], d: int) -> None:
    rng = np.random.default_rng(d)
    low = rng.standard_normal(tuple(s // d for s in shape))
    coords = np.meshgrid(*[np.arange(n) / d - 0.5 + 1 / d / 2 for n in shape], indexing="ij")
    want = scipy.ndimage.map_coordinates(low, coords, order=1, mode="nearest", prefilter=True)
    got = G.add_upsampled(np.zeros(shape), low, d)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
