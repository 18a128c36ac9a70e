"""Many uneven scans in one persistent launch (ScanBatch / SIRTBatch).

Each scan of a batch must get the result of its own one-scan call:
  * projection: bit-identical (the same per-ray code, one thread per ray);
  * backprojection: the same per-voxel sums (rel L2 <= 1e-6 against the
    one-scan kernel with the same voxels-per-thread), and rel L2 <= 1e-5
    against the FP64 oracle for a jittered helical scan;
  * a plan run twice accumulates twice (its counters reset themselves);
  * batches of more than 96 scans (several launches) and empty scans work;
  * SIRTBatch iterations equal per-scan SIRT_flatpanel iterations, eager and
    replayed from a CUDA graph.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import Volume, autotune, geometry, phantoms
from aprict_b200.batch import ScanBatch
from aprict_b200.cb import flatpanel as fp
from aprict_b200.iterators import SIRT_flatpanel, SIRTBatch
from helpers import rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _scans(seed: int, k: int, *, edge=(12, 40), views=(6, 24), det=(16, 56), order="C"):
    rng = np.random.default_rng(seed)
    params = geometry.uneven_scans(rng, k, edge=edge, views=views, det=det, voxwid=1.0, R=150.0, L_minus_R=150.0)
    vols, pgs = [], []
    for i, s in enumerate(params):
        n = s["n"]
        shape = (n, n + i % 3, n + (i % 2) * 2)
        x = phantoms.ellipsoid_volume(seed + i, 4, shape, 1.0, semi_axes_vox=(2, max(3, n // 3)))
        vols.append(Volume(x, voxwid=1.0, order=order, pos_c=(0.3 * i, -0.2 * i, 0.1)))
        pgs.append(geometry.scan_geometry(rng, s))
    return vols, pgs


def test_batched_projection_is_bit_identical() -> None:
    vols, pgs = _scans(1, 7)
    want = []
    for v, pg in zip(vols, pgs):
        ps = fp.ProjectionSet(pg, data=None)
        fp.project(fp.ConfigProject(ssu=2, multiply_before_adding=0.7), v, ps, block=True)
        want.append(ps.data.clone())
    projs = [fp.ProjectionSet(pg, data=None) for pg in pgs]
    ScanBatch(vols, projs).project(fp.ConfigProject(ssu=2, multiply_before_adding=0.7), block=True)
    for p, w in zip(projs, want):
        assert torch.equal(p.data, w)


def test_batched_residual_and_repeat_runs() -> None:
    vols, pgs = _scans(2, 5)
    bases = [torch.rand((pg.num_projs, int(pg.nu.flat[0]), int(pg.nv.flat[0])), device="cuda") for pg in pgs]
    projs = [fp.ProjectionSet(pg, data=None) for pg in pgs]
    plan = ScanBatch(vols, projs).plan_project(fp.ConfigProject(multiply_before_adding=-1), bases=bases)
    plan.run()
    plan.run()  # second run: same result (residual form overwrites), counters reset
    torch.cuda.synchronize()
    for v, pg, b, p in zip(vols, pgs, bases, projs):
        r = fp.ProjectionSet(pg, data=None)
        fp.project_residual(fp.ConfigProject(multiply_before_adding=-1), v, r, b)
        assert torch.equal(p.data, r.data)
    acc = [fp.ProjectionSet(pg, data=None) for pg in pgs]
    plan2 = ScanBatch(vols, acc).plan_project()
    plan2.run()
    plan2.run()
    torch.cuda.synchronize()
    for v, pg, p in zip(vols, pgs, acc):
        one = fp.ProjectionSet(pg, data=None)
        fp.project(fp.ConfigProject(), v, one, block=True)
        assert rel_l2(p.data.cpu().numpy(), 2 * one.data.cpu().numpy()) <= 1e-6


@pytest.mark.parametrize("kw", [dict(fast_approx=True, cyl_mask_rad=9.0, soften_det_edges_proportion=0.05),
                                dict(fast_approx=True, approx_mode_bilinear_interpolate=True),
                                dict()])
def test_batched_backprojection_matches_one_scan_calls(kw) -> None:
    saved = autotune.current()
    autotune.apply({"bp_xb": 0})  # the built-in voxels per thread, as the batch kernel's
    try:
        vols, pgs = _scans(3, 6)
        rng = np.random.default_rng(5)
        projs = [fp.ProjectionSet(pg, data=rng.random((pg.num_projs, int(pg.nu.flat[0]), int(pg.nv.flat[0])),
                                                       dtype=np.float32)) for pg in pgs]
        mults = [Volume(rng.random(v.shape).astype(np.float32) + 0.5, voxwid=1.0, pos_c=v.pos_c) for v in vols]
        cfg = fp.ConfigBackproject(apply_summand_multiplier=True, **kw)
        outs = [v.zeroed_copy() for v in vols]
        ScanBatch(outs, projs).backproject(cfg, multipliers=mults, block=True)
        for v, p, m, o in zip(vols, projs, mults, outs):
            one = v.zeroed_copy()
            fp.backproject(cfg, one, p, summand_multiplier=m, block=True)
            assert np.linalg.norm(one.as_numpy()) > 0
            assert rel_l2(o.as_numpy(), one.as_numpy()) <= 1e-6
    finally:
        autotune.apply(saved)


def test_batched_backprojection_matches_oracle_helical() -> None:
    rng = np.random.default_rng(7)
    s = dict(n=24, views=18, det=40, helical=True, pitch=1.2, pix_at_iso=0.9, voxwid=1.0, R=120.0, L_minus_R=150.0,
             theta0=0.3)
    pg = geometry.scan_geometry(rng, s)
    shape = (24, 26, 22)
    data = rng.random((18, 40, 40), dtype=np.float32)
    cfg = fp.ConfigBackproject(fast_approx=True, cyl_mask_rad=11.0, soften_det_edges_proportion=0.05)
    out = Volume.zeros(shape, voxwid=1.0)
    other = Volume.zeros((10, 10, 10), voxwid=1.0)  # a second scan in the same launch
    p_other = fp.ProjectionSet(fp.ProjGeom.new_circular_scan(num_source_points=5, R=100, L_minus_R=100,
                                                             pix_widhei_at_isocenter=(1, 1), num_pix_widhei=(16, 16)),
                               data=np.ones((5, 16, 16), np.float32))
    ScanBatch([out, other], [fp.ProjectionSet(pg, data=data), p_other]).backproject(cfg, block=True)
    corner = -np.array(shape, np.float32) / 2
    want = O.backproject(pg.to_proj_spec_array(), data, shape, cfg.contents, voxwid=1.0, corner=corner)
    assert rel_l2(out.as_numpy(), want) <= 1e-5


def test_more_than_one_launch_group_and_empty_scans() -> None:
    rng = np.random.default_rng(9)
    vols, projs, want = [], [], []
    for i in range(101):
        n = int(rng.integers(4, 9))
        v = Volume(rng.random((n, n, n)).astype(np.float32), voxwid=1.0)
        m = 0 if i % 25 == 7 else int(rng.integers(1, 4))  # a few scans without views
        pg = fp.ProjGeom.new_circular_scan(num_source_points=max(m, 1), R=40, L_minus_R=40,
                                           pix_widhei_at_isocenter=(0.7, 0.7), num_pix_widhei=(8, 10),
                                           theta_start=0.1 * i)
        if m == 0:
            pg = pg.sliced(slice(0, 0))
        ps = fp.ProjectionSet(pg, data=None)
        one = fp.ProjectionSet(pg, data=None)
        fp.project(fp.ConfigProject(), v, one, block=True)
        vols.append(v)
        projs.append(ps)
        want.append(one.data.clone())
    ScanBatch(vols, projs).project(block=True)
    for p, w in zip(projs, want):
        assert torch.equal(p.data, w)


def _sirt_problems(seed: int, k: int):
    vols, pgs = _scans(seed, k, edge=(16, 32), views=(10, 20), det=(24, 48))
    out = []
    for v, pg in zip(vols, pgs):
        ps = fp.ProjectionSet(pg, data=None)
        fp.project(fp.ConfigProject(), v, ps, block=True)
        out.append((v, pg, ps.data.clone()))
    return out


def test_sirt_batch_equals_individual_sirt() -> None:
    probs = _sirt_problems(11, 4)
    single = [SIRT_flatpanel(SIRT_flatpanel.Config(), v.zeroed_copy(), fp.ProjectionSet(pg, data=b.clone()))
              for v, pg, b in probs]
    batched = [SIRT_flatpanel(SIRT_flatpanel.Config(), v.zeroed_copy(), fp.ProjectionSet(pg, data=b.clone()))
               for v, pg, b in probs]
    for _ in range(3):
        for s in single:
            s.iterate()
    sb = SIRTBatch(batched)
    sb.iterate()
    sb.iterate_graph(2)
    torch.cuda.synchronize()
    for s, t in zip(single, batched):
        assert t.iterations == 3
        assert np.linalg.norm(s.volume.as_numpy()) > 0
        assert rel_l2(t.volume.as_numpy(), s.volume.as_numpy()) <= 1e-6
