"""FORBILD point sampling on the GPU (FBVolume.to_tensor / sample_into) and
the head phantom's known answer.

* against the FP64 oracle (natural-coordinate point tests): identical except
  at sample points within 1e-9 of a surface (none on these grids);
* against the reference's own sampling body (its FP32 _in_region, compiled for
  the CPU): at most 0.2 % of voxels differ (points within FP32 rounding of a
  surface);
* supersampling, accumulation into an existing (F-order) volume;
* the head phantom's projection in priority mode does not overflow the
  covered-interval list (the reference's known answer,
  src/aprict/tests/cuda_kernels/test_project_cb_FORBILD_phantoms.py:120-209:
  1000 helical views, 8 x 8 pixels of 0.1, out_of_mem_count == 0).
"""

from __future__ import annotations

import pathlib

import numpy as np
import pytest
import torch

from aprict_b200 import FBVolume, Volume, phantoms
from aprict_b200.cb import flatpanel as fp
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HEAD = np.load(pathlib.Path(__file__).parent / "golden" / "forbild_head_shapes.npy")


def _grid(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return [np.sort(rng.uniform(lo, hi, k)).astype(np.float32) for k in n]


@pytest.mark.parametrize("which", ["head", "random"])
def test_sampling_matches_oracles(which: str) -> None:
    if which == "head":
        s, (xs, ys, zs) = HEAD, _grid((48, 52, 28), -10.5, 10.5, 1)
    else:
        s = phantoms.random_quadric_phantom(7, n_ellipsoids=40, n_cylinders=30, radius=60)
        xs, ys, zs = _grid((40, 40, 40), -70, 70, 2)
    got = FBVolume(s).to_numpy(xs, ys, zs)
    want = O.forbild_sample(s, xs, ys, zs)
    assert np.abs(want).max() > 0
    assert np.count_nonzero(np.abs(got - want) > 1e-5) == 0
    if O.have_ref():
        ref = O.ref_forbild_sample(s, xs, ys, zs)
        assert (np.abs(got - ref) > 1e-5).mean() <= 2e-3


def test_supersampling_and_accumulate_into_volume() -> None:
    s = phantoms.random_quadric_phantom(9, n_ellipsoids=12, n_cylinders=8, radius=40)
    v = Volume.zeros((30, 34, 26), voxwid=2.7, order="F", pos_c=(1.0, -0.5, 0.25))
    v.fill(0.5)
    FBVolume(s).sample_into(v, supersamp_factor=3)
    xs, ys, zs = v.xs_ys_zs
    want = 0.5 + O.forbild_sample(s, xs, ys, zs, ss_wid=2.7, ss=3)
    got = v.as_numpy()
    assert np.count_nonzero(np.abs(got - want) > 1e-5) <= 2
    assert np.abs(got - want).max() <= 1.0 + 1e-5  # a stray sub-sample moves a voxel by <= |rho| / 27


def test_head_phantom_projection_does_not_overflow() -> None:
    m, n_pix, volres = 1000, 8, 120.0
    ts = np.linspace(0, 2 * np.pi, m, endpoint=False)
    src = np.stack([volres * np.cos(ts), volres * np.sin(ts), (ts - np.pi) / np.pi * volres], axis=1)
    det = np.stack([-volres * np.cos(ts), -volres * np.sin(ts), 0 * ts], axis=1)
    u = np.stack([-0.1 * np.sin(ts), 0.1 * np.cos(ts), 0 * ts], axis=1)
    v = np.broadcast_to(np.array([0.0, 0.0, 0.1]), (m, 3)).copy()
    pg = fp.ProjGeom(source_pos=src, det_pos=det, det_uvec=u, det_vvec=v, nu=n_pix, nv=n_pix)
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), FBVolume(HEAD), ps, block=True)
    assert ps.out_of_mem_count == 0
    assert float(torch.linalg.vector_norm(ps.data)) > 0
    want = O.project_forbild(pg.to_proj_spec_array()[::50], HEAD)
    got = ps.data.cpu().numpy()[::50]
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5
