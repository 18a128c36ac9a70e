"""Element-wise volume kernels vs numpy (float32 semantics of texture_operations.cu)."""

from __future__ import annotations

import numpy as np
import pytest

from aprict_b200 import Volume

pytestmark = pytest.mark.gpu


@pytest.fixture
def arr() -> np.ndarray:
    return np.random.default_rng(0).standard_normal((17, 23, 29)).astype(np.float32)


def test_fill_multiply(arr: np.ndarray) -> None:
    v = Volume(arr, voxwid=1.0)
    v.multiply(2.5)
    np.testing.assert_allclose(v.as_numpy(), arr * np.float32(2.5), rtol=1e-7)
    v.fill(3.25)
    assert np.all(v.as_numpy() == np.float32(3.25))


@pytest.mark.parametrize("order", ["C", "F"])
def test_invert_soft(arr: np.ndarray, order: str) -> None:
    a = np.abs(arr)
    a[0, 0, :5] = 0
    v = Volume(a, voxwid=1.0, order=order)
    v.invert(ignore_zeros=True, softmax_epsilon=0.1)
    want = np.where(a == 0, 0, 1 / (a + 0.1 * np.exp(-a / 0.1)))
    np.testing.assert_allclose(v.as_numpy(), want, rtol=2e-6)


@pytest.mark.parametrize("order", ["C", "F"])
@pytest.mark.parametrize("r0", [0.6, 0.95, 1.0])
def test_softmask_cylinder(arr: np.ndarray, order: str, r0: float) -> None:
    v = Volume(arr, voxwid=1.0, order=order)
    v.soften_to_xy_cylinder(r0)
    X, Y, _ = arr.shape
    ix = np.arange(X)[:, None, None] - (X - 1) / 2
    iy = np.arange(Y)[None, :, None] - (Y - 1) / 2
    rr = np.sqrt(ix**2 + iy**2) / min(X, Y) * 2
    if r0 < 1:
        t = np.clip((rr - r0) / (1 - r0), None, 1)
        m = np.where(rr < r0, 1.0, np.clip((1 + np.cos(np.pi * t)) / 2, 0, 1))
    else:
        m = np.where(rr < 1, 1.0, 0.0)
    np.testing.assert_allclose(v.as_numpy(), arr * m, rtol=1e-5, atol=1e-6)


def test_inner_product_norm(arr: np.ndarray) -> None:
    v = Volume(arr, voxwid=1.0)
    w = Volume(arr[::-1].copy(), voxwid=1.0)
    assert v.inner_product(w) == pytest.approx(float((arr.astype(np.float64) * arr[::-1]).sum()), rel=1e-12)
    assert v.norm == pytest.approx(float(np.linalg.norm(arr.astype(np.float64))), rel=1e-12)


def test_mul_axpy(arr: np.ndarray) -> None:
    v = Volume(arr, voxwid=1.0)
    w = Volume(arr * 2, voxwid=1.0)
    v.add_scaled(w, -0.5)
    np.testing.assert_allclose(v.as_numpy(), np.zeros_like(arr), atol=1e-6)
    v.copy_from(arr)
    v.multiply_volume(w)
    np.testing.assert_allclose(v.as_numpy(), arr * arr * 2, rtol=1e-6)
