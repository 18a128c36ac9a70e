"""Chunked, pipelined drivers for projection stacks kept in host memory (.npy memmaps).

* project_to_array writes exactly what one projection of the whole scan gives
  (bit-identical), for a voxel volume and a FORBILD phantom, with a view count
  that is not a multiple of the chunk size, and matches the FP64 oracle
  (rel L2 <= 1e-5; the chunked driver of src/aprict/scripts/project_cbfp.py:335-470);
* with photons_per_pixel the chunks carry Poisson noise of the right size;
* backproject_from_array equals one all-view backprojection (rel L2 <= 1e-6,
  chunks summed in order) and the FP64 oracle's backprojection (<= 1e-5).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import FBVolume, Volume, phantoms
from aprict_b200.cb import flatpanel as fp
from aprict_b200.outofcore import backproject_from_array, project_to_array
from helpers import circular, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_project_to_memmap_equals_one_call(tmp_path) -> None:
    pg = circular(37, 120, 120, 0.537, 40, 36)
    vol = Volume(phantoms.ellipsoid_volume(2, 5, (32, 30, 28), 1.0, semi_axes_vox=(3, 10)), voxwid=1.0)
    one = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), vol, one, block=True)
    out = np.lib.format.open_memmap(tmp_path / "p.npy", "w+", dtype=np.float32, shape=(37, 40, 36))
    assert project_to_array(fp.ConfigProject(), vol, pg, out, views_per_chunk=8) == 0
    np.testing.assert_array_equal(np.asarray(out), one.data.cpu().numpy())
    want, _ = O.project_siddon(pg.to_proj_spec_array(), vol.as_numpy(), voxwid=1.0,
                               corner=-np.array((32, 30, 28), np.float32) / 2)
    assert rel_l2(np.asarray(out), want) <= 1e-5
    fb = FBVolume(phantoms.random_quadric_phantom(3, n_ellipsoids=6, n_cylinders=4, radius=20))
    one = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), fb, one, block=True)
    out2 = np.zeros((37, 40, 36), np.float32)
    project_to_array(fp.ConfigProject(), fb, pg, out2, views_per_chunk=5)
    np.testing.assert_array_equal(out2, one.data.cpu().numpy())
    assert rel_l2(out2, O.project_forbild(pg.to_proj_spec_array(), fb.shapes)) <= 1e-5


def test_noise() -> None:
    pg = circular(12, 120, 120, 0.537, 32, 32)
    vol = Volume(phantoms.ellipsoid_volume(4, 4, (24, 24, 24), 1.0, semi_axes_vox=(3, 8)), voxwid=1.0)
    clean = np.zeros((12, 32, 32), np.float32)
    noisy = np.zeros_like(clean)
    project_to_array(fp.ConfigProject(), vol, pg, clean, views_per_chunk=5)
    project_to_array(fp.ConfigProject(), vol, pg, noisy, views_per_chunk=5, photons_per_pixel=1e4, seed=3)
    d = noisy - clean
    sd = np.sqrt(np.exp(clean) / 1e4)  # std of -log(Poisson(I0 e^-p)/I0) ~ sqrt(e^p / I0)
    assert abs(np.mean(d / sd)) < 0.1 and 0.8 < np.std(d / sd) < 1.2


def test_backproject_from_memmap_equals_one_call(tmp_path) -> None:
    pg = circular(41, 120, 120, 0.537, 40, 44)
    data = np.random.default_rng(1).random((41, 40, 44), dtype=np.float32)
    path = tmp_path / "q.npy"
    np.save(path, data)
    mm = np.load(path, mmap_mode="r")
    cfg = fp.ConfigBackproject(fast_approx=True)
    a = Volume.zeros((30, 32, 34), voxwid=1.0)
    b = Volume.zeros((30, 32, 34), voxwid=1.0)
    fp.backproject(cfg, a, fp.ProjectionSet(pg, data=torch.from_numpy(data).cuda()), block=True)
    backproject_from_array(cfg, b, pg, mm, views_per_chunk=9)
    assert np.linalg.norm(a.as_numpy()) > 0
    assert rel_l2(b.as_numpy(), a.as_numpy()) <= 1e-6
    want = O.backproject(pg.to_proj_spec_array(), data, (30, 32, 34), cfg.contents, voxwid=1.0,
                         corner=-np.array((30, 32, 34), np.float32) / 2)
    assert rel_l2(b.as_numpy(), want) <= 1e-5
