"""aprict_b200_batch_run_static: the batch run whose work counters live in the
library's static device array (for callers that cannot allocate).

Called through the C ABI and compared with aprict_b200_batch_run on two calls
in a row (the counters must be clean for the second call), for a projection
plan and an accumulating backprojection plan, and for a plan of more than 96
scans (several launch groups, whose counters sit further into the array); a
plan with more launch groups than the array holds is rejected before anything
is enqueued. This file is
collected last so that it also runs after every other GPU test.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import Volume, _lib, geometry, phantoms
from aprict_b200.batch import ScanBatch
from aprict_b200.cb import flatpanel as fp
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _scans(seed: int, k: int):
    rng = np.random.default_rng(seed)
    params = geometry.uneven_scans(rng, k, edge=(12, 32), views=(6, 20), det=(16, 48), voxwid=1.0, R=150.0,
                                   L_minus_R=150.0)
    vols, pgs = [], []
    for i, s in enumerate(params):
        n = s["n"]
        vols.append(Volume(phantoms.ellipsoid_volume(seed + i, 4, (n, n, n), 1.0, semi_axes_vox=(2, max(3, n // 3))),
                           voxwid=1.0))
        pgs.append(geometry.scan_geometry(rng, s))
    return vols, pgs


def _run_static(plan) -> None:
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().aprict_b200_batch_run_static(plan._host.ctypes.data, stream), "batch_run_static")


def _run_existing(plan) -> None:
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().aprict_b200_batch_run(plan._host.ctypes.data, plan._dev.data_ptr(), stream), "batch_run")


def test_static_scratch_projection_matches_batch_run() -> None:
    vols, pgs = _scans(31, 6)
    bases = [torch.rand((pg.num_projs, int(pg.nu.flat[0]), int(pg.nv.flat[0])), device="cuda") for pg in pgs]
    a = [fp.ProjectionSet(pg, data=None) for pg in pgs]
    b = [fp.ProjectionSet(pg, data=None) for pg in pgs]
    cfg = fp.ConfigProject(multiply_before_adding=-1)
    plan_a = ScanBatch(vols, a).plan_project(cfg, bases=bases)
    plan_b = ScanBatch(vols, b).plan_project(cfg, bases=bases)
    for _ in range(2):
        _run_static(plan_a)
        _run_existing(plan_b)
        torch.cuda.synchronize()
        for pa, pb in zip(a, b):
            assert np.linalg.norm(pb.data.cpu().numpy()) > 0
            assert rel_l2(pa.data.cpu().numpy(), pb.data.cpu().numpy()) <= 1e-6


def test_static_scratch_backprojection_matches_batch_run_twice() -> None:
    vols, pgs = _scans(32, 5)
    rng = np.random.default_rng(3)
    projs = [fp.ProjectionSet(pg, data=rng.random((pg.num_projs, int(pg.nu.flat[0]), int(pg.nv.flat[0])),
                                                   dtype=np.float32)) for pg in pgs]
    cfg = fp.ConfigBackproject(fast_approx=True, soften_det_edges_proportion=0.05)
    out_a = [v.zeroed_copy() for v in vols]
    out_b = [v.zeroed_copy() for v in vols]
    plan_a = ScanBatch(out_a, projs).plan_backproject(cfg)
    plan_b = ScanBatch(out_b, projs).plan_backproject(cfg)
    for call in range(2):  # accumulating: the second call adds the same again
        _run_static(plan_a)
        _run_existing(plan_b)
        torch.cuda.synchronize()
        for va, vb in zip(out_a, out_b):
            assert np.linalg.norm(vb.as_numpy()) > 0
            assert rel_l2(va.as_numpy(), vb.as_numpy()) <= 1e-6, call


def test_static_scratch_several_launch_groups_twice() -> None:
    # 130 small scans = 2 launch groups; each call must start from cleared
    # counters in both groups' slots (a plan whose counters were left non-zero
    # by a foreign write would skip work units)
    rng = np.random.default_rng(34)
    vols, projs_a, projs_b = [], [], []
    for i in range(130):
        n = int(rng.integers(4, 10))
        vols.append(Volume(rng.random((n, n, n)).astype(np.float32), voxwid=1.0))
        pg = fp.ProjGeom.new_circular_scan(num_source_points=int(rng.integers(1, 5)), R=40, L_minus_R=40,
                                           pix_widhei_at_isocenter=(0.7, 0.7), num_pix_widhei=(8, 10),
                                           theta_start=0.1 * i)
        projs_a.append(fp.ProjectionSet(pg, data=None))
        projs_b.append(fp.ProjectionSet(pg, data=None))
    plan_a = ScanBatch(vols, projs_a).plan_project()
    plan_b = ScanBatch(vols, projs_b).plan_project()
    assert plan_a._host[:32].view(np.int32)[4] >= 2  # n_groups
    for call in range(2):  # accumulating projections: the second call adds the same again
        _run_static(plan_a)
        _run_existing(plan_b)
        torch.cuda.synchronize()
        for pa, pb in zip(projs_a, projs_b):
            assert np.linalg.norm(pb.data.cpu().numpy()) > 0
            assert rel_l2(pa.data.cpu().numpy(), pb.data.cpu().numpy()) <= 1e-6, call


def test_static_scratch_rejects_too_many_groups() -> None:
    # A host plan header claiming 16 launch groups (> the 15 the array holds):
    # rejected before any device call.
    vols, pgs = _scans(33, 1)
    plan = ScanBatch(vols, [fp.ProjectionSet(pgs[0], data=None)]).plan_project()
    fake = plan._host.copy()
    hdr = fake[:32].view(np.int32)
    hdr[4] = 16  # n_groups
    with pytest.raises(_lib.AprictError, match="static scratch holds at most 15 groups"):
        _lib.check(_lib.lib().aprict_b200_batch_run_static(fake.ctypes.data, None), "batch_run_static")
