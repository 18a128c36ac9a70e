"""Siddon forward projector on the GPU vs the FP64 oracle and the reference.

Gate: rel L2 <= 1e-5 against the FP64 oracle (the stated tolerance for
projections). Agreement with the reference's own kernel (compiled for the CPU,
FP32 with incremental stepping) is reported and loosely bounded: the reference
is the less accurate of the two (its own error vs FP64 is ~5e-6).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import Volume, phantoms
from aprict_b200.cb import flatpanel as fp
from helpers import circular, jittered, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _run(vol_np: np.ndarray, pg: fp.ProjGeom, *, voxwid: float = 1.0, order: str = "C", pos_c=(0, 0, 0), **cfg) -> np.ndarray:
    v = Volume(vol_np, voxwid=voxwid, order=order, pos_c=pos_c)
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(**cfg), v, ps, block=True)
    return ps.data.cpu().numpy()


def _oracle(vol_np, pg, *, voxwid=1.0, pos_c=(0, 0, 0), svf=1.0, mba=1.0, ssu=1, ssv=1):
    corner = np.asarray(pos_c, np.float32) - np.float32(voxwid) * np.array(vol_np.shape, np.float32) / 2
    out, _ = O.project_siddon(pg.to_proj_spec_array(), vol_np, voxwid=voxwid, corner=corner, svf=svf, mba=mba, ssu=ssu, ssv=ssv)
    return out


@pytest.fixture(scope="module")
def vol48() -> np.ndarray:
    return phantoms.ellipsoid_volume(3, 8, (48, 40, 36), 1.0, semi_axes_vox=(3, 14))


def test_matches_oracle_circular(vol48: np.ndarray) -> None:
    pg = circular(24, 120, 120, 0.5, 80, 64)
    got = _run(vol48, pg)
    want = _oracle(vol48, pg)
    assert np.linalg.norm(want) > 0
    assert rel_l2(got, want) <= TOL


def test_matches_reference(vol48: np.ndarray) -> None:
    if not O.have_ref():
        pytest.skip("reference oracle not built")
    pg = circular(12, 120, 120, 0.5, 64, 48)
    got = _run(vol48, pg)
    corner = -np.array(vol48.shape, np.float32) / 2
    ref = O.ref_project_siddon(pg.to_proj_spec_array(), vol48, voxwid=1.0, corner=corner)
    want = _oracle(vol48, pg)
    e_ref = rel_l2(ref, want)
    e_ours = rel_l2(got, want)
    print(f"rel L2 vs FP64: ours {e_ours:.2e}  reference {e_ref:.2e}; ours vs reference {rel_l2(got, ref):.2e}")
    assert rel_l2(got, ref) <= 5e-5
    assert e_ours <= e_ref * 1.5 + 1e-7


@pytest.mark.parametrize("order", ["C", "F"])
def test_orders_and_offcentre(vol48: np.ndarray, order: str) -> None:
    pg = circular(10, 150, 90, 0.7, 40, 56, theta0=0.3)
    got = _run(vol48, pg, voxwid=1.3, order=order, pos_c=(3.0, -2.0, 5.5))
    want = _oracle(vol48, pg, voxwid=1.3, pos_c=(3.0, -2.0, 5.5))
    assert rel_l2(got, want) <= TOL


def test_jittered_arbitrary_geometry(vol48: np.ndarray) -> None:
    rng = np.random.default_rng(7)
    pg = jittered(rng, circular(16, 110, 130, 0.6, 48, 40))
    got = _run(vol48, pg)
    want = _oracle(vol48, pg)
    assert rel_l2(got, want) <= TOL


@pytest.mark.parametrize(("ssu", "ssv", "svf", "mba"), [(2, 1, 1.0, 1.0), (3, 2, 1.0, -1.0), (1, 1, 1.5, 2.5)])
def test_supersampling_shrink_multiply(vol48: np.ndarray, ssu: int, ssv: int, svf: float, mba: float) -> None:
    pg = circular(8, 120, 120, 0.5, 32, 24)
    got = _run(vol48, pg, ssu=ssu, ssv=ssv, shrink_volume_factor=svf, multiply_before_adding=mba)
    want = _oracle(vol48, pg, ssu=ssu, ssv=ssv, svf=svf, mba=mba)
    assert rel_l2(got, want) <= TOL


def test_supersampling_invariant(vol48: np.ndarray) -> None:
    """ssu x ssv supersampled projection == box-downsampled fine-detector projection
    (metamorphic check of src/aprict/tests/cuda_kernels/test_project_cb_FORBILD_supersampling.py:300-324)."""
    ssu, ssv = 2, 3
    pg = circular(6, 120, 120, 0.6, 24, 20)
    coarse = _run(vol48, pg, ssu=ssu, ssv=ssv)
    fine_pg = fp.ProjGeom(
        source_pos=pg.source_pos,
        det_pos=pg.det_pos,
        det_uvec=pg.det_uvec / ssu,
        det_vvec=pg.det_vvec / ssv,
        nu=pg.nu * ssu,
        nv=pg.nv * ssv,
    )
    fine = _run(vol48, fine_pg)
    down = fine.reshape(6, 24, ssu, 20, ssv).mean(axis=(2, 4))
    assert rel_l2(coarse, down) <= 1e-5


def test_accumulates_and_residual(vol48: np.ndarray) -> None:
    pg = circular(6, 120, 120, 0.5, 32, 32)
    v = Volume(vol48, voxwid=1.0)
    base = torch.rand((6, 32, 32), device="cuda")
    ps = fp.ProjectionSet(pg, data=base.clone())
    fp.project(fp.ConfigProject(), v, ps, block=True)
    ax = _oracle(vol48, pg)
    assert rel_l2(ps.data.cpu().numpy() - base.cpu().numpy(), ax) <= 1e-5
    # fused residual: r = b - A x in one pass
    r = fp.ProjectionSet(pg, data=None)
    fp.project_residual(fp.ConfigProject(multiply_before_adding=-1), v, r, base)
    torch.cuda.synchronize()
    assert rel_l2(r.data.cpu().numpy(), base.cpu().numpy() - ax) <= 1e-5


def test_leading_dims_and_strides(vol48: np.ndarray) -> None:
    pg1 = circular(5, 120, 120, 0.5, 20, 16)
    pg = fp.ProjGeom(
        source_pos=np.stack([pg1.source_pos, pg1.source_pos[::-1]]),
        det_pos=np.stack([pg1.det_pos, pg1.det_pos[::-1]]),
        det_uvec=np.stack([pg1.det_uvec, pg1.det_uvec[::-1]]),
        det_vvec=np.broadcast_to(pg1.det_vvec, (2, 5, 3)).copy(),
        nu=20,
        nv=16,
    )
    assert pg.projs_list_shape == (2, 5)
    big = torch.zeros((2, 5, 20, 32), device="cuda")
    data = big[..., ::2]  # v stride 2
    ps = fp.ProjectionSet(pg, data=data)
    fp.project(fp.ConfigProject(), Volume(vol48, voxwid=1.0), ps, block=True)
    want = _oracle(vol48, pg1)
    got = data.cpu().numpy()
    assert rel_l2(got[0], want) <= TOL
    assert rel_l2(got[1], want[::-1]) <= TOL
    assert float(big[..., 1::2].abs().max()) == 0.0


def test_fan_beam_single_row() -> None:
    """nv == 1 (fan beam): rays lie in the z = 0 plane through voxel centres."""
    vol = phantoms.ellipsoid_volume(5, 6, (64, 64, 1), 0.5, semi_axes_vox=(3, 12))
    pg = circular(30, 60, 50, 0.4, 96, 1)
    got = _run(vol, pg, voxwid=0.5)
    want = _oracle(vol, pg, voxwid=0.5)
    assert np.linalg.norm(want) > 0
    assert rel_l2(got, want) <= TOL


def test_constant_cube_path_length() -> None:
    """A unit-density cube: each line integral equals the chord length through the cube."""
    n = 32
    vol = np.ones((n, n, n), np.float32)
    pg = circular(8, 80, 80, 0.5, 48, 48)
    got = _run(vol, pg)
    specs = pg.to_proj_spec_array()
    # analytic chord length of each pixel-centre ray through [-16,16]^3
    s = np.stack([specs["source_pos"][k] for k in "xyz"], -1)[:, None, None, :].astype(np.float64)
    P = np.stack([specs["det_pos"][k] for k in "xyz"], -1).astype(np.float64)
    U = np.stack([specs["det_u"][k] for k in "xyz"], -1).astype(np.float64)
    V = np.stack([specs["det_v"][k] for k in "xyz"], -1).astype(np.float64)
    iu = np.arange(48) - 23.5
    p = P[:, None, None, :] + U[:, None, None, :] * iu[None, :, None, None] + V[:, None, None, :] * iu[None, None, :, None]
    d = p - s
    with np.errstate(divide="ignore", invalid="ignore"):
        t0 = (-16 - s) / d
        t1 = (16 - s) / d
    lo = np.nanmax(np.minimum(t0, t1), axis=-1).clip(0, 1)
    hi = np.nanmin(np.maximum(t0, t1), axis=-1).clip(0, 1)
    want = np.clip(hi - lo, 0, None) * np.linalg.norm(d, axis=-1)
    assert np.abs(got - want).max() <= 1e-4 * want.max()


def test_rays_missing_volume_give_zero() -> None:
    vol = np.ones((8, 8, 8), np.float32)
    pg = circular(4, 100, 100, 0.5, 16, 16)
    got = _run(vol, pg, pos_c=(0, 0, 500.0))  # volume far above every ray
    assert float(np.abs(got).max()) == 0.0


def test_empty_projection_set_is_noop() -> None:
    vol = np.ones((8, 8, 8), np.float32)
    pg = circular(1, 100, 100, 0.5, 4, 4)
    pg_empty = pg.sliced([])
    ps = fp.ProjectionSet(pg_empty, data=None)
    fp.project(fp.ConfigProject(), Volume(vol, voxwid=1.0), ps, block=True)
    assert ps.data.numel() == 0
