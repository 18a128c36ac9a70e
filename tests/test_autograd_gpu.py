"""Differentiable projector: torch autograd with the matched-adjoint backward.

Checks (the differentiable-SIRT workload's checks, at test size):
  * dot-product test <A x, y> == <x, A^T y> to 1e-6;
  * autograd gradient of 0.5 ||A x - b||^2 == A^T (A x - b) from the FP64 oracle;
  * central finite differences on 64 random voxels (h = 1e-3);
  * equal to the reference's own Landweber gradient, its exact backprojection of
    the residual (src/aprict/iterators/landweber_vram.py:221-260 with
    --exact-adjoint), run on the CPU;
  * double backward gives the Hessian-vector product A^T A v.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import phantoms
from aprict_b200.autograd import SiddonProjector
from aprict_b200.cb import flatpanel as fp
from helpers import circular, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPE = (36, 40, 32)


@pytest.fixture(scope="module")
def setup():
    pg = circular(24, 100, 100, 0.537, 48, 44)
    proj = SiddonProjector(pg, SHAPE, voxwid=1.0)
    xt = torch.from_numpy(phantoms.ellipsoid_volume(7, 6, SHAPE, 1.0, semi_axes_vox=(3, 12))).cuda()
    b = proj.forward_raw(xt) + 0.01 * torch.randn(proj.data_shape, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    return pg, proj, xt, b


def test_dot_product(setup) -> None:
    pg, proj, _, _ = setup
    g = torch.Generator("cuda").manual_seed(1)
    x = torch.rand(SHAPE, device="cuda", generator=g)
    y = torch.rand(proj.data_shape, device="cuda", generator=g)
    lhs = float((proj.forward_raw(x).double() * y.double()).sum())
    rhs = float((x.double() * proj.adjoint_raw(y).double()).sum())
    assert abs(lhs - rhs) / abs(lhs) <= 1e-6


def test_gradient_matches_oracle_and_reference(setup) -> None:
    pg, proj, xt, b = setup
    x = (0.7 * xt).clone().requires_grad_(True)
    loss = 0.5 * ((proj(x) - b).double() ** 2).sum()
    loss.backward()
    grad = x.grad.cpu().numpy()
    r = (proj.forward_raw(x.detach()) - b).cpu().numpy()
    corner = -np.array(SHAPE, np.float32) / 2
    want = O.backproject_transpose(pg.to_proj_spec_array(), r, SHAPE, voxwid=1.0, corner=corner)
    assert rel_l2(grad, want) <= 1e-5
    if O.have_ref():
        ref = np.zeros(SHAPE, np.float32)
        O.ref_backproject(pg.to_proj_spec_array(), r, ref, fp.ConfigBackproject().contents, voxwid=1.0, corner=corner)
        assert rel_l2(grad, ref) <= 1e-5


def test_central_finite_differences(setup) -> None:
    _, proj, xt, b = setup
    x0 = (0.8 * xt).clone()
    x = x0.clone().requires_grad_(True)
    (0.5 * ((proj(x) - b).double() ** 2).sum()).backward()
    grad = x.grad.double()

    def loss(v: torch.Tensor) -> float:
        return float(0.5 * ((proj.forward_raw(v) - b).double() ** 2).sum())

    rng = np.random.default_rng(3)
    h = 1e-3
    idx = [tuple(int(rng.integers(8, s - 8)) for s in SHAPE) for _ in range(64)]
    fd, an = [], []
    for i in idx:
        xp = x0.clone()
        xm = x0.clone()
        xp[i] += h
        xm[i] -= h
        fd.append((loss(xp) - loss(xm)) / (2 * h))
        an.append(float(grad[i]))
    fd, an = np.array(fd), np.array(an)
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) <= 2e-3


def test_double_backward_hessian_vector(setup) -> None:
    _, proj, xt, b = setup
    x = (0.5 * xt).clone().requires_grad_(True)
    loss = 0.5 * ((proj(x) - b) ** 2).sum()
    (g,) = torch.autograd.grad(loss, x, create_graph=True)
    v = torch.rand(SHAPE, device="cuda", generator=torch.Generator("cuda").manual_seed(4))
    (hv,) = torch.autograd.grad((g * v).sum(), x)
    want = proj.adjoint_raw(proj.forward_raw(v))
    assert rel_l2(hv.cpu().numpy(), want.cpu().numpy()) <= 1e-5


def test_gradient_descent_reduces_loss(setup) -> None:
    _, proj, _, b = setup
    x = torch.zeros(SHAPE, device="cuda", requires_grad=True)
    opt = torch.optim.SGD([x], lr=1e-4)
    losses = []
    for _ in range(5):
        opt.zero_grad()
        loss = 0.5 * ((proj(x) - b) ** 2).sum()
        loss.backward()
        opt.step()
        losses.append(float(loss))
    assert losses[-1] < losses[0]
