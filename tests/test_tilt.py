"""The tilted (cone-cylinder) projection filter on the CPU.

* The oracle's order-1 "grid-constant" rotation against scipy.ndimage.rotate
  itself -- the published definition behind the reference's
  cupyx.scipy.ndimage.rotate calls (src/aprict/cb/ramp_filter.py:667-679,
  790-806) -- with and without the zero padding of the filter's frame.
* The oracle's taps against the product's (pinned to the reference's golden
  vectors in test_ramp.py).
* The host side of FBPFilterer's tilted path against the oracle: padded frame,
  largest angle, letterbox columns, weight mask and the rotation-angle draws
  (one rng.random() per projection, ramp_filter.py:443-460).
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.ndimage
import scipy.special

from aprict_b200 import ramp_kernels
from aprict_b200.cb.ramp_filter import FBPFilterer
from oracle import tilt as T


@pytest.mark.parametrize("angle", [0.0, 3.7, -11.25, 45.0, 90.0, -137.0])
@pytest.mark.parametrize("shape", [(37, 23), (16, 16), (40, 1)])
def test_oracle_rotation_is_scipy_rotate(angle: float, shape: tuple[int, int]) -> None:
    rng = np.random.default_rng(abs(int(angle * 10)) + shape[0])
    img = rng.standard_normal(shape)
    want = scipy.ndimage.rotate(img, angle, axes=(1, 0), reshape=False, order=1, mode="grid-constant", prefilter=False)
    c, s = scipy.special.cosdg(angle), scipy.special.sindg(angle)
    got = T.rotate(img, c, s, shape, ((shape[0] - 1) / 2, (shape[1] - 1) / 2))
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


def test_oracle_rotation_with_padding_and_crop() -> None:
    rng = np.random.default_rng(3)
    img = rng.standard_normal((30, 12))
    padx, pady = 4, 2
    big = np.pad(img, ((padx, padx), (pady, pady)))
    centre = ((big.shape[0] - 1) / 2, (big.shape[1] - 1) / 2)
    c, s = scipy.special.cosdg(-7.5), scipy.special.sindg(-7.5)
    want = scipy.ndimage.rotate(big, -7.5, axes=(1, 0), reshape=False, order=1, mode="grid-constant", prefilter=False)
    got = T.rotate(img, c, s, big.shape, centre, in_off=(padx, pady))
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
    # rotating back into the unpadded window is the crop of the full back-rotation
    back_full = scipy.ndimage.rotate(want, 7.5, axes=(1, 0), reshape=False, order=1, mode="grid-constant", prefilter=False)
    cb, sb = scipy.special.cosdg(7.5), scipy.special.sindg(7.5)
    back = T.rotate(want, cb, sb, img.shape, centre, out_off=(padx, pady))
    np.testing.assert_allclose(back, back_full[padx:-padx, pady:-pady], rtol=0, atol=1e-12)


def test_oracle_taps_match_product_taps() -> None:
    for n, pw in [(7, 1.0), (63, 0.37), (2 * 200 - 1, 0.0021)]:
        np.testing.assert_allclose(T.ramlak_taps(n, pw), ramp_kernels.ramp_kernel_ramlak(n, pw), rtol=1e-13, atol=0)
        np.testing.assert_array_equal(T.hilbert_taps(n), ramp_kernels.hilbert_transform_kernel(n))


def _bare(nu: int, nv: int, pw: float, L: float, zeta: float | None = None, seed: int = 0) -> FBPFilterer:  # noqa: N803
    """An FBPFilterer with only its host state (no device buffers), for CPU tests."""
    f = FBPFilterer.__new__(FBPFilterer)
    f.L, f.physpixwid, f.proj_2d_shape = L, pw, (nu, nv)
    f._max_abs_rotation_angle = zeta if zeta is not None else FBPFilterer.get_max_abs_rotation_angle((nu, nv), pw, L)
    f._expanded_2d_shape = FBPFilterer.get_expanded_proj_2d_shape((nu, nv), f._max_abs_rotation_angle)
    f.rng = np.random.default_rng(seed)
    return f


@pytest.mark.parametrize(("nu", "nv", "pw", "L"), [(384, 384, 0.8, 1000.0), (100, 31, 1.3, 700.0), (64, 64, 2.0, 90.0)])
def test_frame_letterbox_and_draws(nu: int, nv: int, pw: float, L: float) -> None:  # noqa: N803
    f = _bare(nu, nv, pw, L, seed=11)
    zeta = T.max_rotation_angle(nu, nv, pw, L)
    assert f.zeta == zeta
    assert f._expanded_2d_shape == T.expanded_shape(nu, nv, zeta, hacky=False)
    assert FBPFilterer.get_expanded_proj_2d_shape((nu, nv), zeta, _hacky_fdk_mode=True) == (nu, nv)
    nv_e = f._expanded_2d_shape[1]
    for ang in np.linspace(-zeta, zeta, 9).astype(np.float32)[1:-1]:
        np.testing.assert_array_equal(f._letterbox_columns(ang), T.letterbox_columns(ang, zeta, L, pw, nv_e))
    # all views at once (the filter's path): the per-view values, bit for bit
    many = _bare(nu, nv, pw, L, seed=5).uniform_rng(-zeta, zeta, 2000)
    np.testing.assert_array_equal(f._letterbox_matrix(many), np.stack([f._letterbox_columns(a) for a in many]))
    with pytest.raises(ValueError):
        f._letterbox_matrix(np.array([0.0, 1.01 * zeta + 1e-3]))
    with pytest.raises(ValueError):
        f.get_letterbox_slice(1.01 * zeta + 1e-3)
    draws = f.uniform_rng(-zeta, zeta, 25)
    np.testing.assert_array_equal(draws, T.uniform_angles(np.random.default_rng(11), -zeta, zeta, 25))
    f.advance_rng(3)
    r = np.random.default_rng(11)
    for _ in range(28):
        r.random()
    assert f.rng.random() == r.random()


@pytest.mark.parametrize("fdk", [False, True])
def test_weight_mask_follows_reference_chain(fdk: bool) -> None:
    from aprict_b200.cb.ramp_filter import frame_weight_mask

    for shape, pw, L in [((50, 21), 0.9, 300.0), ((401, 384), 0.8, 1000.0)]:  # noqa: N806
        got = frame_weight_mask(shape, pw, L, fdk)
        assert got.dtype == np.float64 and got.shape == shape
        np.testing.assert_array_equal(got, T.weight_mask(*shape, pw, L, fdk))
