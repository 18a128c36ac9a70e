"""FORBILD analytic projection: the FP64 oracle vs the reference, the host shape
compiler, and the GPU kernel vs both.

Gates: GPU vs FP64 oracle rel L2 <= 1e-5 (projections). The reference computes
its intervals in FP32, so GPU vs reference is bounded at 1e-4.
"""

from __future__ import annotations

import numpy as np
import pytest

from aprict_b200 import _structs as S
from aprict_b200 import phantoms
from aprict_b200.cb import forbild
from helpers import circular, random_shapes_all_types, rel_l2
from oracle import oracle as O

TYPES_REF = (1, 2, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16)  # type 5 below


def test_interval_oracle_matches_reference_all_types() -> None:
    if not O.have_ref():
        pytest.skip("reference oracle not built")
    rng = np.random.default_rng(0)
    shapes = random_shapes_all_types(rng, 150, types=TYPES_REF)
    worst = 0.0
    for _ in range(300):
        v1 = rng.uniform(-120, 120, 3)
        v2 = rng.uniform(-120, 120, 3)
        for s in shapes:
            a = O.forbild_interval(v1, v2, s)
            b = O.ref_forbild_interval(v1, v2, s)
            la = 0.0 if a is None else a[1] - a[0]
            lb = max(0.0, b[1] - b[0])
            worst = max(worst, abs(la - lb))
    assert worst <= 2e-5, worst


def test_cone_z_offcentre_reference_quirk_documented() -> None:
    """Cone_z (type 5) away from z = 0: the reference's cull projects the ray
    direction with z = pos.z instead of 0 (FORBILD_volumes.h, FORBILD_Cone_z
    clip), so it can wrongly reject rays; the oracle and the GPU kernel keep the
    exact frustum. Centred at z = 0 both agree."""
    if not O.have_ref():
        pytest.skip("reference oracle not built")
    rng = np.random.default_rng(5)
    shapes = random_shapes_all_types(rng, 40, types=(5,))
    shapes["z"] = 0.0
    for s in shapes:
        s["cas1"]["mode"] = s["cas2"]["mode"] = s["cas3"]["mode"] = 0
    worst = 0.0
    for _ in range(300):
        v1 = rng.uniform(-120, 120, 3)
        v2 = rng.uniform(-120, 120, 3)
        for s in shapes:
            a = O.forbild_interval(v1, v2, s)
            b = O.ref_forbild_interval(v1, v2, s)
            worst = max(worst, abs((0.0 if a is None else a[1] - a[0]) - max(0.0, b[1] - b[0])))
    assert worst <= 2e-5


@pytest.mark.parametrize("overlap_addition", [False, True])
def test_projection_oracle_matches_reference(overlap_addition: bool) -> None:
    if not O.have_ref():
        pytest.skip("reference oracle not built")
    rng = np.random.default_rng(1)
    shapes = random_shapes_all_types(rng, 48, types=TYPES_REF)
    pg = circular(6, 150, 150, 0.5, 40, 36)
    specs = pg.to_proj_spec_array()
    ref, ovf = O.ref_project_forbild(specs, shapes, overlap_addition=overlap_addition)
    ora = O.project_forbild(specs, shapes, mode=1 if overlap_addition else 0)
    assert ovf == 0
    assert np.linalg.norm(ora) > 0
    assert rel_l2(ref, ora) <= 1e-4


def test_compile_shapes() -> None:
    rng = np.random.default_rng(2)
    shapes = random_shapes_all_types(rng, 32)
    q = forbild.compile_shapes(shapes)
    assert q.dtype == S.quadric and len(q) == 32
    kinds = {1: 4, 2: 3, 3: 3, 4: 3, 5: 3, 6: 2, 7: 2, 8: 2, 9: 2, 10: 1, 11: 1, 12: 2, 13: 1, 14: 2, 15: 2, 16: 2}
    assert all(q["kind"][i] == kinds[int(shapes["type"][i])] for i in range(32))
    # bounding boxes contain points sampled from the shapes (oracle in-region test via tiny segments)
    lo, hi = forbild.shape_bboxes(shapes)
    for i in range(32):
        c = np.array([shapes["x"][i], shapes["y"][i], shapes["z"][i]], np.float64)
        assert np.all(lo[i] <= c) and np.all(c <= hi[i])
    bad = shapes[:1].copy()
    bad["type"] = 40
    with pytest.raises(ValueError, match="unknown type"):
        forbild.compile_shapes(bad)
    bad["type"] = 13
    bad["r"] = -1
    with pytest.raises(ValueError, match="invalid parameters"):
        forbild.compile_shapes(bad)


def test_fbvolume_bbox_and_prune() -> None:
    from aprict_b200 import FBVolume

    sh = phantoms.random_quadric_phantom(3, n_ellipsoids=10, n_cylinders=5)
    v = FBVolume(sh)
    lo, hi = v.get_bbox()
    assert np.all(lo < hi)
    assert len(v.prune_to_bbox(lo, hi).shapes) == 15
    assert len(v.prune_to_bbox((1e4, 1e4, 1e4), (2e4, 2e4, 2e4)).shapes) == 0


# ---------------------------------------------------------------- GPU
def _gpu_project(shapes, pg, **cfg):
    from aprict_b200 import FBVolume
    from aprict_b200.cb import flatpanel as fp

    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(**cfg), FBVolume(shapes), ps, block=True)
    return ps.data.cpu().numpy(), ps.out_of_mem_count


@pytest.mark.gpu
@pytest.mark.parametrize(
    ("mode_kw", "mode"),
    [({}, 0), ({"overlap_addition": True}, 1), ({"overlap_addition": True, "additive_line_integral": True}, 2)],
)
def test_gpu_matches_oracle_all_types(mode_kw: dict, mode: int) -> None:
    rng = np.random.default_rng(11)
    shapes = random_shapes_all_types(rng, 64)
    pg = circular(8, 150, 150, 0.5, 64, 48)
    got, ovf = _gpu_project(shapes, pg, **mode_kw)
    want = O.project_forbild(pg.to_proj_spec_array(), shapes, mode=mode)
    assert ovf == 0
    assert np.linalg.norm(want) > 0
    assert rel_l2(got, want) <= 1e-5


@pytest.mark.gpu
def test_gpu_supersampling_multiply_and_chunks() -> None:
    """More shapes than one shared-memory chunk (96), ssu/ssv > 1, mba != 1."""
    rng = np.random.default_rng(12)
    shapes = random_shapes_all_types(rng, 200, radius=60)
    pg = circular(4, 150, 150, 0.5, 48, 40)
    got, _ = _gpu_project(shapes, pg, ssu=2, ssv=3, multiply_before_adding=-1.5)
    want = O.project_forbild(pg.to_proj_spec_array(), shapes, mode=0, ssu=2, ssv=3, mba=-1.5)
    assert rel_l2(got, want) <= 1e-5


@pytest.mark.gpu
def test_gpu_matches_reference_quadric_phantom() -> None:
    if not O.have_ref():
        pytest.skip("reference oracle not built")
    shapes = phantoms.random_quadric_phantom(4, n_ellipsoids=12, n_cylinders=8, radius=60)
    pg = circular(6, 200, 150, 0.4, 64, 64)
    for kw, ovl in (({}, False), ({"overlap_addition": True}, True)):
        got, _ = _gpu_project(shapes, pg, **kw)
        ref, _ = O.ref_project_forbild(pg.to_proj_spec_array(), shapes, overlap_addition=ovl)
        assert rel_l2(got, ref) <= 1e-4


@pytest.mark.gpu
def test_gpu_fan_and_empty() -> None:
    rng = np.random.default_rng(13)
    shapes = random_shapes_all_types(rng, 20)
    pg = circular(10, 150, 150, 0.5, 96, 1)
    got, _ = _gpu_project(shapes, pg)
    want = O.project_forbild(pg.to_proj_spec_array(), shapes, mode=0)
    assert rel_l2(got, want) <= 1e-5
    empty = shapes[:0]
    got0, _ = _gpu_project(empty, pg)
    assert float(np.abs(got0).max()) == 0.0
