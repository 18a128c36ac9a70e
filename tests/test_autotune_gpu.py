"""Launch-shape knobs change speed only: every knob value gives the same result.

The forward projector computes each ray independently of the tile it sits in,
so its output is bit-identical across tile heights, warp patch shapes and
views per tile. The backprojector's wave
size only reorders CTAs, so it is bit-identical too; its voxels-per-thread
count changes where the per-view affine terms are stepped from (a thread's
first voxel), so results across that knob agree to float rounding (rel L2
1e-6). The autotuner must pick allowed values and leave its inputs untouched.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import Volume, autotune, phantoms
from aprict_b200.cb import flatpanel as fp
from helpers import circular, rel_l2

pytestmark = pytest.mark.gpu

SHAPE = (40, 36, 44)


@pytest.fixture()
def restore_knobs():
    saved = autotune.current()
    yield
    autotune.apply(saved)


def _problem():
    vol = Volume(phantoms.ellipsoid_volume(5, 6, SHAPE, 1.0, semi_axes_vox=(3, 12)), voxwid=1.0)
    pg = circular(16, 120, 120, 0.537, 52, 56)
    return vol, pg


def test_projector_tile_shapes_are_bit_identical(restore_knobs) -> None:
    vol, pg = _problem()
    outs = []
    for tv in autotune.FP_TILE_V:
        for wv in autotune.FP_WARP_V:
            for tw, ww in autotune.FP_VIEWS:
                autotune.apply({"fp_tile_v": tv, "fp_warp_v": wv, "fp_views": tw, "fp_warp_views": ww})
                ps = fp.ProjectionSet(pg, data=None)
                fp.project(fp.ConfigProject(ssu=2), vol, ps, block=True)
                outs.append(ps.data.cpu().numpy())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    # an odd view count leaves the last multi-view tile part empty; the
    # ray-driven adjoint shares the tiles (atomic sums: equal to rounding)
    pg5 = circular(5, 120, 120, 0.537, 52, 56)
    y = fp.ProjectionSet(pg5, data=np.random.default_rng(3).random((5, 52, 56), dtype=np.float32))
    outs, adj = [], []
    for tw, ww in autotune.FP_VIEWS:
        autotune.apply({"fp_views": tw, "fp_warp_views": ww})
        ps = fp.ProjectionSet(pg5, data=None)
        fp.project(fp.ConfigProject(), vol, ps, block=True)
        outs.append(ps.data.cpu().numpy())
        v = Volume.zeros(SHAPE, voxwid=1.0)
        fp.backproject_adjoint(fp.ConfigProject(), v, y, block=True)
        adj.append(v.as_numpy())
    for o, a in zip(outs[1:], adj[1:]):
        assert np.array_equal(o, outs[0])
        assert rel_l2(a, adj[0]) <= 1e-6
    assert np.linalg.norm(adj[0]) > 0


@pytest.mark.parametrize("kw", [dict(), dict(fast_approx=True, approx_mode_bilinear_interpolate=True), dict(fast_approx=True)])
def test_backprojector_shapes_are_bit_identical(restore_knobs, kw) -> None:
    vol, pg = _problem()
    rng = np.random.default_rng(2)
    ps = fp.ProjectionSet(pg, data=rng.random((16, 52, 56), dtype=np.float32))
    cfg = fp.ConfigBackproject(**kw)
    by_xb = {}
    for xb in autotune.BP_XB:
        outs = []
        for wave in (1, 3, 7):
            autotune.apply({"bp_xb": xb, "bp_wave": wave})
            v = Volume.zeros(SHAPE, voxwid=1.0)
            fp.backproject(cfg, v, ps, block=True)
            outs.append(v.data.cpu().numpy())
        for o in outs[1:]:
            assert np.array_equal(o, outs[0])
        by_xb[xb] = outs[0]
    assert np.linalg.norm(by_xb[4]) > 0
    assert rel_l2(by_xb[2], by_xb[4]) <= 1e-6


def test_tune_picks_allowed_values_and_caches(restore_knobs, tmp_path) -> None:
    vol, pg = _problem()
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), vol, ps, block=True)
    before_p = ps.data.clone()
    before_v = vol.data.clone()
    cache = tmp_path / "tune.json"
    choice = autotune.tune(ps, vol, cfg_bp=fp.ConfigBackproject(), cache_file=cache)
    assert choice["fp_tile_v"] in autotune.FP_TILE_V and choice["fp_warp_v"] in autotune.FP_WARP_V
    assert (choice["fp_views"], choice["fp_warp_views"]) in autotune.FP_VIEWS
    assert choice["bp_xb"] in autotune.BP_XB and choice["bp_wave"] in autotune.BP_WAVE
    assert autotune.current()["fp_tile_v"] == choice["fp_tile_v"]
    assert torch.equal(ps.data, before_p) and torch.equal(vol.data, before_v)
    assert cache.exists()
    autotune.apply({})
    assert autotune.tune(ps, vol, cfg_bp=fp.ConfigBackproject(), cache_file=cache) == choice
