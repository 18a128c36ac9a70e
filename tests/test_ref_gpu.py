"""The reference's own GPU kernels, launched as the reference launches them.

oracle/_ref/libaprict_refgpu.so compiles the reference's projector and
backprojector kernel files unchanged for sm_100a; the bench times them beside
ours. These checks pin that launcher: on a small non-cubic volume, the
reference's kernels on the GPU give what the same kernel source gives compiled
for the CPU (oracle/_ref/libaprict_ref.so, one host thread per CUDA thread), and
agree with this library's kernels to the reference's own FP32 accuracy.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import Volume, phantoms
from aprict_b200.cb import flatpanel as fp
from helpers import circular, rel_l2
from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not O.have_ref_gpu(), reason="reference GPU kernels not built")]

SHAPE = (24, 20, 16)


@pytest.fixture(scope="module")
def problem():
    pg = circular(12, 60.0, 60.0, 0.537, 32, 28)
    x = phantoms.ellipsoid_volume(5, 5, SHAPE, 1.0, semi_axes_vox=(2, 7))
    corner = -np.array(SHAPE, np.float32) / 2
    return pg, x, corner


def test_reference_gpu_projection(problem) -> None:
    pg, x, corner = problem
    ps = fp.ProjectionSet(pg, data=None)
    specs_dev = ps.specs_device()
    out = torch.zeros((pg.num_projs, 32, 28), dtype=torch.float32, device="cuda")
    vol = O.RefGpuVolume(torch.from_numpy(x).cuda().contiguous())
    O.ref_gpu_project(vol, specs_dev.data_ptr(), pg.num_projs, 32, 28, out, voxwid=1.0, corner=corner)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    cpu = O.ref_project_siddon(pg.to_proj_spec_array(), x, voxwid=1.0, corner=corner)
    assert np.linalg.norm(cpu) > 0
    assert rel_l2(got, cpu) <= 1e-5
    ours = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), Volume(x, voxwid=1.0), ours, block=True)
    assert rel_l2(got, ours.data.cpu().numpy()) <= 1e-4
    vol.close()


@pytest.mark.parametrize("kw", [dict(fast_approx=True, cyl_mask_rad=9.0, soften_det_edges_proportion=0.05), dict()],
                         ids=["fast", "exact"])
def test_reference_gpu_backprojection(problem, kw) -> None:
    pg, x, corner = problem
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), Volume(x, voxwid=1.0), ps, block=True)
    data = ps.data.contiguous()
    mult = (np.random.default_rng(2).random(SHAPE).astype(np.float32) + 0.5)
    cfg = fp.ConfigBackproject(apply_summand_multiplier=True, **kw)
    vol = O.RefGpuVolume(torch.zeros(SHAPE, dtype=torch.float32, device="cuda"))
    mvol = O.RefGpuVolume(torch.from_numpy(mult).cuda().contiguous())
    O.ref_gpu_backproject(vol, pg.to_proj_spec_array(), data, cfg.contents, voxwid=1.0, corner=corner, mult=mvol)
    back = torch.empty(SHAPE, dtype=torch.float32, device="cuda")
    vol.read(back)
    torch.cuda.synchronize()
    got = back.cpu().numpy()
    cpu = np.zeros(SHAPE, np.float32)
    O.ref_backproject(pg.to_proj_spec_array(), data.cpu().numpy(), cpu, cfg.contents, voxwid=1.0, corner=corner,
                      mult=mult)
    assert np.linalg.norm(cpu) > 0
    assert rel_l2(got, cpu) <= 1e-5
    ours = Volume.zeros(SHAPE, voxwid=1.0)
    fp.backproject(cfg, ours, ps, summand_multiplier=Volume(mult, voxwid=1.0), block=True)
    assert rel_l2(got, ours.as_numpy()) <= 1e-4
    vol.close()
    mvol.close()
