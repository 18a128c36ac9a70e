"""The tilted (cone-cylinder) FBP filter and driver on the GPU vs the FP64 oracle.

* ``aprict_b200_rotate_projections`` against the oracle's rotation with the
  library's float32 roundings: equal up to the rounding of an FP64 sum
  (forward: padding, weight mask, letterbox; back: crop).
* FBPFilterer's tilted path (random angles drawn as the reference draws them,
  forced angles, the Hilbert output, the chunked generator) against the oracle
  filter: rel L2 <= 1e-5 (FP32 convolution vs FP64).
* fbp_cone_cyl (one- and two-sided) against the oracle driver built from the
  oracle filter and the FP64 backprojection oracle: rel L2 <= 1e-4.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import Volume, _lib, phantoms
from aprict_b200.cb import flatpanel as fp
from aprict_b200.cb.ramp_filter import FBPFilterer
from aprict_b200.recon import fbp_cone_cyl
from helpers import rel_l2
from oracle import oracle as O
from oracle import tilt as T

pytestmark = pytest.mark.gpu


def _desc(t: torch.Tensor) -> np.ndarray:
    return _lib.proj_desc(tuple(t.shape), tuple(t.stride()))


def _rotate(src: torch.Tensor, out: torch.Tensor, cs: np.ndarray, centre, in_off, out_off, mask=None, colw=None) -> None:
    cs_d = torch.from_numpy(np.ascontiguousarray(cs, np.float64)).cuda()
    m_d = None if mask is None else torch.from_numpy(np.ascontiguousarray(mask, np.float64)).cuda()
    c_d = None if colw is None else torch.from_numpy(np.ascontiguousarray(colw, np.float64)).cuda()
    d_src, d_out = _desc(src), _desc(out)
    _lib.check(_lib.lib().aprict_b200_rotate_projections(
        _lib.ptr(d_src), src.data_ptr(), _lib.ptr(d_out), out.data_ptr(), cs_d.data_ptr(), centre[0], centre[1],
        in_off[0], in_off[1], out_off[0], out_off[1], None if m_d is None else m_d.data_ptr(),
        None if c_d is None else c_d.data_ptr(), torch.cuda.current_stream().cuda_stream), "rotate_projections")
    torch.cuda.synchronize()


def test_rotate_kernel_matches_oracle() -> None:
    rng = np.random.default_rng(1)
    m, nu, nv, padx, pady = 6, 45, 17, 5, 1
    nu_e, nv_e = nu + 2 * padx, nv + 2 * pady
    centre = ((nu_e - 1) / 2, (nv_e - 1) / 2)
    x = rng.standard_normal((m, nu, nv)).astype(np.float32)
    angles = np.array([0.0, 0.031, -0.2, 0.7, -1.3, 2.9], np.float32)
    cs = np.array([T.rotation_cs(-180 / np.pi * a) for a in angles])
    mask = rng.uniform(0.5, 1.0, (nu_e, nv_e))
    colw = rng.uniform(0.0, 1.0, (m, nv_e))
    out = torch.empty((m, nu_e, nv_e), device="cuda")
    _rotate(torch.from_numpy(x).cuda(), out, cs, centre, (padx, pady), (0, 0), mask, colw)
    got = out.cpu().numpy()
    want = np.stack([
        ((T.rotate(x[i], *cs[i], (nu_e, nv_e), centre, in_off=(padx, pady)).astype(np.float32).astype(np.float64)
          * mask).astype(np.float32).astype(np.float64) * colw[i][None, :]).astype(np.float32)
        for i in range(m)
    ])
    np.testing.assert_allclose(got, want, rtol=2e-7, atol=1e-30)
    assert np.count_nonzero(got != want) <= got.size // 1000
    np.testing.assert_array_equal(got[0], want[0])  # angle 0: pure pad, mask and letterbox

    # back-rotation into the unpadded window (crop), strided output
    big = torch.zeros((m, nu + 3, nv), device="cuda")
    dst = big[:, 1 : nu + 1, :]
    _rotate(out, dst, np.array([T.rotation_cs(180 / np.pi * a) for a in angles]), centre, (0, 0), (padx, pady))
    back = dst.cpu().numpy()
    want_b = np.stack([T.rotate(got[i], *T.rotation_cs(180 / np.pi * angles[i]), (nu, nv), centre, out_off=(padx, pady))
                       for i in range(m)]).astype(np.float32)
    np.testing.assert_allclose(back, want_b, rtol=2e-7, atol=1e-30)
    assert float(big[:, 0].abs().max()) == 0 and float(big[:, nu + 1 :].abs().max()) == 0


def _filter_case(nu=56, nv=20, pw=1.1, L=400.0, m=9):  # noqa: N803
    rng = np.random.default_rng(nu + nv)
    x = rng.random((m, nu, nv)).astype(np.float32)
    return x, pw, L


@pytest.mark.parametrize("hilbert", [False, True])
def test_filter_random_angles_matches_oracle(hilbert: bool) -> None:
    x, pw, L = _filter_case()  # noqa: N806
    m, nu, nv = x.shape
    f = FBPFilterer(L=L, physpixwid=pw, proj_2d_shape=(nu, nv), include_hilbert_transform_in_output=hilbert,
                    rng=np.random.default_rng(5))
    outs, _ = f.filter_bulk_axis1_concat(torch.from_numpy(x).cuda())
    angles = T.uniform_angles(np.random.default_rng(5), -f.zeta, f.zeta, m)
    want = T.filter_tilted(x, L=L, physpixwid=pw, angles=angles, zeta=f.zeta, hilbert=hilbert)
    assert len(outs) == len(want) == (2 if hilbert else 1)
    for g, w in zip(outs, want):
        assert np.linalg.norm(w) > 0
        assert rel_l2(g.cpu().numpy(), w) <= 1e-5


def test_filter_forced_angle_stream_and_limit_zeta() -> None:
    x, pw, L = _filter_case(nu=40, nv=16, m=7)  # noqa: N806
    m, nu, nv = x.shape
    f = FBPFilterer(L=L, physpixwid=pw, proj_2d_shape=(nu, nv), limit_zeta=0.01, projs_per_batch=3,
                    rng=np.random.default_rng(2))
    assert f.zeta == 0.01
    ang = np.float64(-0.0071)
    (got,), _ = f.filter_bulk_axis1_concat(x, force_rotation_angle=ang)
    want = T.filter_tilted(x, L=L, physpixwid=pw, angles=ang * np.ones((m,), np.float32), zeta=0.01)[0]
    assert rel_l2(got.cpu().numpy(), want) <= 1e-5
    # the generator draws the same angles chunk by chunk
    g = FBPFilterer(L=L, physpixwid=pw, proj_2d_shape=(nu, nv), limit_zeta=0.01, projs_per_batch=3,
                    rng=np.random.default_rng(2))
    parts = [o[0].cpu().numpy() for o, _ in g.filter_bulk_axis1_stream(torch.from_numpy(x).cuda())]
    assert [p.shape[0] for p in parts] == [3, 3, 1]
    (whole,), _ = f.__class__(L=L, physpixwid=pw, proj_2d_shape=(nu, nv), limit_zeta=0.01,
                              rng=np.random.default_rng(2)).filter_bulk_axis1_concat(x)
    np.testing.assert_array_equal(np.concatenate(parts), whole.cpu().numpy())


def _golden_theta_scan(m: int, R: float, LmR: float, pix: float, nu: int, nv: int, h: float) -> fp.ProjGeom:  # noqa: N803
    """Cylindrical golden-angle trajectory of the reference's cone-cyl geometries
    (make_geometry_cone_cyl.py:233-289): z evenly spaced, theta steps of (sqrt 5 - 1) pi."""
    zs = np.linspace(-h / 2, h / 2, num=m + 2, endpoint=True)[1:-1]
    ts = 0.3 + np.arange(m) * (np.sqrt(5) - 1) * np.pi
    src = np.stack([R * np.cos(ts), R * np.sin(ts), zs], axis=1)
    det = np.stack([-LmR * np.cos(ts), -LmR * np.sin(ts), zs], axis=1)
    u = pix * np.stack([-np.sin(ts), np.cos(ts), 0 * ts], axis=1)
    v = np.broadcast_to(pix * np.array([0.0, 0.0, -1.0]), (m, 3)).copy()
    return fp.ProjGeom(source_pos=src, det_pos=det, det_uvec=u, det_vvec=v, nu=nu, nv=nv)


@pytest.mark.parametrize("two_sided", [False, True])
def test_fbp_cone_cyl_matches_oracle(two_sided: bool) -> None:
    n, vw = 24, 1.0
    R, LmR, pix, nu, nv = 90.0, 90.0, 1.6, 40, 24  # noqa: N806
    m = 60
    pg = _golden_theta_scan(m, R, LmR, pix, nu, nv, h=30.0)
    x = phantoms.ellipsoid_volume(4, 6, (n, n, n), vw, semi_axes_vox=(2, 8))
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), Volume(x, voxwid=vw), ps, block=True)
    out = Volume.zeros((n, n, n), voxwid=vw)
    fbp_cone_cyl(ps, out, two_sided=two_sided, seed_proj_rots=9, num_projs_per_chunk=16)
    got = out.as_numpy()

    L = R + LmR  # noqa: N806
    zeta = T.max_rotation_angle(nu, nv, pix, L)
    angles = T.uniform_angles(np.random.default_rng(9), -zeta, zeta, m)
    corner = -np.array((n, n, n), np.float32) * np.float32(vw / 2)
    specs = pg.to_proj_spec_array()

    def bp(sp, data, cfg):
        return O.backproject(sp, data, (n, n, n), fp.ConfigBackproject(**cfg).contents, voxwid=vw, corner=corner)

    support = R * np.sin(np.arctan(pix * nu / 2 / L))
    zs = pg.source_pos[:, 2]
    want = T.fbp_cone_cyl(specs, ps.data.cpu().numpy(), (n, n, n), vw, corner, R=R, L=L, pixwid=pix, zeta=zeta,
                          angles=angles, two_sided=two_sided, cyl_mask_rad=support, zs_span=float(zs.max() - zs.min()),
                          backproject=bp)
    assert np.linalg.norm(want) > 0
    assert rel_l2(got, want) <= 1e-4
