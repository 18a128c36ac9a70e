"""float16 volumes and float16 / float64 projections on the GPU.

The reference instantiates its projector and backprojector for half and float
volumes and half, float and double projections (src/aprict/cb/flatpanel.py:
120-185); its kernels compute in float. Here the kernels compute in FP32 on
converted working copies, so every result equals the FP32 path on the
converted inputs: bit for bit where the output is FP32 or FP64, rounded once
where the output is float16.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import FBVolume, Volume, phantoms
from aprict_b200.cb import flatpanel as fp
from aprict_b200.iterators import SIRT_flatpanel
from helpers import circular

pytestmark = pytest.mark.gpu

SHAPE = (24, 20, 16)


def _geom() -> fp.ProjGeom:
    return circular(18, 80.0, 70.0, 0.9, 32, 24)


def _vol(dtype) -> tuple[np.ndarray, Volume]:
    x = phantoms.ellipsoid_volume(5, 6, SHAPE, 1.0, semi_axes_vox=(2, 6)).astype(dtype)
    return x, Volume(x, voxwid=1.0, order="F")


def test_half_volume_ops_round_the_fp32_results() -> None:
    x, v = _vol(np.float16)
    assert v.dtype == np.float16 and v.data.dtype == torch.float16
    ops = [lambda vol: vol.multiply(1.7), lambda vol: vol.soften_to_xy_cylinder(0.8),
           lambda vol: vol.invert(ignore_zeros=True, softmax_epsilon=0.1)]
    for op in ops:  # each op: the FP32 op on the current values, rounded once to float16
        ref = Volume(v.as_numpy().astype(np.float32), voxwid=1.0, order="F")
        op(v)
        op(ref)
        np.testing.assert_array_equal(v.as_numpy(), ref.as_numpy().astype(np.float16))
    assert abs(v.inner_product(v) - float((v.as_numpy().astype(np.float64) ** 2).sum())) <= 1e-9 * v.inner_product(v)
    w = Volume.zeros(SHAPE, voxwid=1.0, dtype=np.float16)
    w.fill(2.0)
    assert w.as_numpy().dtype == np.float16 and np.all(w.as_numpy() == 2.0)


def test_project_half_volume_into_double_and_half_projections() -> None:
    pg = _geom()
    x, vh = _vol(np.float16)
    v32 = Volume(x.astype(np.float32), voxwid=1.0, order="F")
    p32 = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), v32, p32, block=True)
    want = p32.data.double()
    rng = np.random.default_rng(1)
    start = torch.from_numpy(rng.random(tuple(p32.data.shape))).cuda()
    p64 = fp.ProjectionSet(pg, data=start.clone())
    fp.project(fp.ConfigProject(), vh, p64, block=True)
    assert p64.data.dtype == torch.float64
    assert torch.equal(p64.data, start + want)  # accumulated in FP64
    p16 = fp.ProjectionSet(pg, data=None)
    p16.create_buffer(dtype=np.float16)
    fp.project(fp.ConfigProject(), vh, p16, block=True)
    assert p16.data.dtype == torch.float16 and torch.equal(p16.data, p32.data.half())


def test_forbild_into_double_projections() -> None:
    pg = _geom()
    shapes = phantoms.random_quadric_phantom(2, n_ellipsoids=4, n_cylinders=2, radius=12)
    p32 = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), FBVolume(shapes), p32, block=True)
    p64 = fp.ProjectionSet(pg, data=None)
    p64.create_buffer(dtype=np.float64)
    fp.project(fp.ConfigProject(), FBVolume(shapes), p64, block=True)
    assert torch.equal(p64.data, p32.data.double()) and float(p32.data.abs().max()) > 0


@pytest.mark.parametrize("fast", [True, False])
def test_backproject_double_projections_into_half_volume(fast: bool) -> None:
    pg = _geom()
    rng = np.random.default_rng(2)
    y64 = torch.from_numpy(rng.random((18, 32, 24))).cuda()
    x = rng.random(SHAPE).astype(np.float16)
    vh = Volume(x, voxwid=1.0)
    v32 = Volume(x.astype(np.float32), voxwid=1.0)
    m = rng.uniform(0.5, 1.5, SHAPE).astype(np.float16)
    cfg = fp.ConfigBackproject(fast_approx=fast, apply_summand_multiplier=True, cyl_mask_rad=9.0)
    fp.backproject(cfg, vh, fp.ProjectionSet(pg, data=y64), summand_multiplier=Volume(m, voxwid=1.0), block=True)
    fp.backproject(cfg, v32, fp.ProjectionSet(pg, data=y64.float()),
                   summand_multiplier=Volume(m.astype(np.float32), voxwid=1.0), block=True)
    assert vh.data.dtype == torch.float16
    np.testing.assert_array_equal(vh.as_numpy(), v32.as_numpy().astype(np.float16))


def test_sirt_with_double_measurement() -> None:
    pg = _geom()
    x, v32 = _vol(np.float32)
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), v32, ps, block=True)
    xa, xb = Volume.zeros(SHAPE, voxwid=1.0), Volume.zeros(SHAPE, voxwid=1.0)
    sa = SIRT_flatpanel(SIRT_flatpanel.Config(), xa, fp.ProjectionSet(pg, data=ps.data.clone()))
    sb = SIRT_flatpanel(SIRT_flatpanel.Config(), xb, fp.ProjectionSet(pg, data=ps.data.double()))
    for _ in range(3):
        sa.iterate()
        sb.iterate()
    torch.cuda.synchronize()
    assert np.linalg.norm(xa.as_numpy()) > 0
    np.testing.assert_array_equal(xb.as_numpy(), xa.as_numpy())
