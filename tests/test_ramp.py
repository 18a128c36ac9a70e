"""Ramp filtering: tap formulas vs the reference's golden vectors, and the GPU convolution kernel.

CPU tests pin the taps (src/aprict/ramp_kernels.py:43-59) against the
known-answer vectors of src/aprict/tests/ramp_kernels/test_ramp_kernels_precision.py:33-147
(extracted by tests/golden/make_ramp_golden.py). GPU tests compare the filter
kernels (the shared-memory FFT convolution for rows of 128 to 2048 samples, the
direct convolution otherwise) with an FP64 numpy convolution: gate rel L2
<= 1e-5, and the golden vectors within FP32 accuracy.
"""

from __future__ import annotations

import json
import pathlib

import numpy as np
import pytest

from aprict_b200 import ramp_kernels

GOLDEN = json.loads((pathlib.Path(__file__).parent / "golden" / "ramlak_golden.json").read_text())


def conv_same_fp64(x: np.ndarray, taps: np.ndarray) -> np.ndarray:
    """out[m] = sum_j taps[m - j + nu - 1] x[j] (taps of length 2 nu - 1), in float64."""
    nu = x.shape[-1]
    full = np.convolve(np.asarray(x, np.float64), np.asarray(taps, np.float64), mode="full")
    return full[nu - 1 : 2 * nu - 1]


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=[c["id"] for c in GOLDEN["cases"]])
def test_ramlak_taps_reproduce_golden(case: dict) -> None:
    """Pin the tap formula with the reference test's own procedure.

    The golden outputs are what scipy's FFT convolution of the float32 input
    with float64 taps returns (test_ramp_kernels_precision.py:162-175); the
    FFT of a float32 array runs in single precision, so they sit ~1e-6 from
    the exact convolution. Re-running that procedure with our taps must
    reproduce them to ~1e-14 (any tap error would show), and the exact FP64
    convolution must agree to within that single-precision rounding.
    """
    import scipy.signal

    x = np.array(case["input"], dtype=np.float32)
    n = len(x)
    taps = ramp_kernels.ramp_kernel_ramlak(2 * n + 1, 1.0)
    want = np.array(case["expected"])
    got = scipy.signal.convolve(x, taps.astype(np.float64), mode="same", method="fft")
    assert np.linalg.norm(got - want) <= 1e-12 * max(1.0, np.linalg.norm(want))
    exact = np.convolve(x.astype(np.float64), taps, mode="full")[n : 2 * n]
    assert np.linalg.norm(exact - want) <= 1e-5 * max(1.0, np.linalg.norm(want))


def test_tap_formulas() -> None:
    h = ramp_kernels.ramp_kernel_ramlak(9, 0.5)
    k = np.arange(-4, 5).astype(float)
    want = np.zeros(9)
    want[k == 0] = np.pi**2
    odd = k % 2 != 0
    want[odd] = -4.0 / k[odd] ** 2
    np.testing.assert_allclose(h, want / 0.5, rtol=1e-14, atol=1e-14)
    assert ramp_kernels.odd_only(h)
    assert not ramp_kernels.odd_only(ramp_kernels.apodize_hann(h))
    hil = ramp_kernels.hilbert_transform_kernel(7)
    np.testing.assert_allclose(hil, [2 / -3, 2 / -2, 2 / -1, 0, 2, 1, 2 / 3])
    with pytest.raises(ValueError, match="odd"):
        ramp_kernels.ramp_kernel(8)
    # Hann apodisation multiplies the response by (1 + cos 2 pi f)/2
    n = 1025
    taps = ramp_kernels.ramp_kernel_ramlak(n, 1.0)
    H = np.fft.rfft(np.roll(np.pad(taps, (0, 4096 - n)), -(n // 2)))  # noqa: N806
    Ha = np.fft.rfft(np.roll(np.pad(ramp_kernels.apodize_hann(taps), (0, 4096 - n)), -(n // 2)))  # noqa: N806
    f = np.arange(len(H)) / 4096
    np.testing.assert_allclose(Ha.real[1:-1], (H * 0.5 * (1 + np.cos(2 * np.pi * f))).real[1:-1], rtol=0, atol=1e-2 * np.abs(H).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN["cases"], ids=[c["id"] for c in GOLDEN["cases"]])
def test_gpu_filter_golden(case: dict) -> None:
    import torch

    from aprict_b200.cb.ramp_filter import RampFilterer

    x = np.array(case["input"], dtype=np.float32)
    n = len(x)
    rf = RampFilterer(physpixwid=1.0, proj_2d_shape=(n, 1), projs_per_batch=1)
    (out,) = rf.filter(torch.from_numpy(x.reshape(1, n, 1)).cuda())
    got = out.cpu().numpy().reshape(n).astype(np.float64)
    want = np.array(case["expected"])
    # FP32 kernel: the reference's own FP32 FFT path is 1.3e-6 off on the step case
    assert np.linalg.norm(got - want) <= 2e-5 * max(1.0, np.linalg.norm(want))


@pytest.mark.gpu
@pytest.mark.parametrize(("nu", "nv", "apod", "hilbert"), [(1024, 1, None, False), (300, 7, "hann", False), (96, 33, None, True), (17, 1, "hann", True)])
def test_gpu_filter_matches_fp64(nu: int, nv: int, apod: str | None, hilbert: bool) -> None:
    import torch

    from aprict_b200.cb.ramp_filter import RampFilterer

    rng = np.random.default_rng(nu)
    m = 5
    data = rng.random((m, nu, nv)).astype(np.float32)
    w = rng.random((nu, nv)).astype(np.float32)
    funcs = (ramp_kernels.ramp_kernel_ramlak,) + ((ramp_kernels.hilbert_transform_kernel,) if hilbert else ())
    rf = RampFilterer(physpixwid=0.37, proj_2d_shape=(nu, nv), override_kern_funcs=funcs, apodization=apod)
    outs = rf.filter(torch.from_numpy(data).cuda(), weights=torch.from_numpy(w).cuda(), scale=0.5)
    for taps, out in zip(rf.taps, outs):
        want = 0.5 * np.stack(
            [np.stack([conv_same_fp64(data[i, :, j] * w[:, j].astype(np.float64), taps) for j in range(nv)], -1) for i in range(m)]
        )
        got = out.cpu().numpy()
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= 1e-5, err


@pytest.mark.gpu
def test_gpu_filter_strided_views() -> None:
    import torch

    from aprict_b200.cb.ramp_filter import RampFilterer

    rng = np.random.default_rng(2)
    big = torch.from_numpy(rng.random((6, 64, 10)).astype(np.float32)).cuda()
    view = big[::2, :, 1::3]  # (3, 64, 3) non-contiguous
    rf = RampFilterer(physpixwid=1.0, proj_2d_shape=(64, 3))
    (out,) = rf.filter(view)
    taps = rf.taps[0]
    v = view.cpu().numpy()
    want = np.stack([np.stack([conv_same_fp64(v[i, :, j], taps) for j in range(3)], -1) for i in range(3)])
    assert np.linalg.norm(out.cpu().numpy() - want) / np.linalg.norm(want) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("nu", [127, 128, 129, 257, 438, 1000, 2048, 2049])
@pytest.mark.parametrize("layout", ["u_rows", "v_rows", "strided"])
def test_gpu_filter_sizes_and_layouts(nu: int, layout: str) -> None:
    """Rows of 128 to 2048 samples take the FFT convolution (FP64 forward
    transform, two rows per complex signal), shorter and longer ones the direct
    convolution: both against the FP64 convolution, for rows contiguous along u
    or v, strided views, an odd row count (the last complex signal carries one
    row) and asymmetric taps (Hilbert at half-pixel offset)."""
    import torch

    from aprict_b200.cb.ramp_filter import RampFilterer

    rng = np.random.default_rng(nu + len(layout))
    m, nv = 3, 5
    if layout == "u_rows":
        data = torch.from_numpy(rng.random((m, nv, nu)).astype(np.float32)).cuda().permute(0, 2, 1)
    elif layout == "v_rows":
        data = torch.from_numpy(rng.random((m, nu, nv)).astype(np.float32)).cuda()
    else:
        big = torch.from_numpy(rng.random((2 * m, nu, 2 * nv + 1)).astype(np.float32)).cuda()
        data = big[::2, :, 1::2]
    w = torch.from_numpy(rng.random((nu, nv)).astype(np.float32) + 0.5).cuda()
    funcs = (ramp_kernels.ramp_kernel_ramlak, ramp_kernels.hilbert_transform_kernel_halfoffset)
    rf = RampFilterer(physpixwid=0.41, proj_2d_shape=(nu, nv), override_kern_funcs=funcs, apodization="hann")
    outs = [torch.zeros_like(data) for _ in funcs] if layout != "strided" else None
    outs = rf.filter(data, weights=w, scale=0.75, outs=outs)
    d = data.cpu().numpy().astype(np.float64) * w.cpu().numpy().astype(np.float64)[None]
    for taps, out in zip(rf.taps, outs):
        want = 0.75 * np.stack([np.stack([conv_same_fp64(d[i, :, j], taps) for j in range(nv)], -1) for i in range(m)])
        err = np.linalg.norm(out.cpu().numpy() - want) / np.linalg.norm(want)
        assert err <= 1e-5, err


@pytest.mark.gpu
def test_gpu_fft_entry_points_match_direct_through_the_c_abi() -> None:
    """aprict_b200_ramp_fft_tables + aprict_b200_ramp_filter_fft against
    aprict_b200_ramp_filter on the same rows, taps and weights, called through
    ctypes as a C caller would: the tables built once, the filter run twice
    (the tables are not consumed), rows along v with an odd row count."""
    import torch

    from aprict_b200 import _lib

    lib = _lib.lib()
    rng = np.random.default_rng(11)
    m, nu, nv = 5, 700, 3  # 15 rows: the last complex signal carries one
    x = torch.from_numpy(rng.random((m, nu, nv)).astype(np.float32)).cuda()
    w = torch.from_numpy(rng.random((nu, nv)).astype(np.float32) + 0.5).cuda()
    taps = torch.from_numpy(ramp_kernels.apodize_hann(ramp_kernels.ramp_kernel_ramlak(2 * nu - 1, 0.3)).astype(np.float32)).cuda()
    nbytes = int(lib.aprict_b200_ramp_fft_tables_bytes(nu))
    assert nbytes == 32 * 2048
    tables = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.aprict_b200_ramp_fft_tables(taps.data_ptr(), nu, tables.data_ptr(), st), "ramp_fft_tables")
    d = _lib.proj_desc(tuple(x.shape), tuple(x.stride()))
    want = torch.empty_like(x)
    _lib.check(
        lib.aprict_b200_ramp_filter(_lib.ptr(d), x.data_ptr(), _lib.ptr(d), want.data_ptr(), taps.data_ptr(), 0,
                                    w.data_ptr(), w.stride(0), w.stride(1), 0.25, st),
        "ramp_filter",
    )
    for _ in range(2):
        got = torch.full_like(x, float("nan"))
        _lib.check(
            lib.aprict_b200_ramp_filter_fft(_lib.ptr(d), x.data_ptr(), _lib.ptr(d), got.data_ptr(), tables.data_ptr(),
                                            w.data_ptr(), w.stride(0), w.stride(1), 0.25, st),
            "ramp_filter_fft",
        )
        torch.cuda.synchronize()
        assert torch.isfinite(got).all()
        err = (torch.linalg.norm((got - want).double()) / torch.linalg.norm(want.double())).item()
        assert err <= 1e-5, err
