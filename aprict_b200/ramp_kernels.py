"""1-D filter taps for filtered backprojection (drop-in for ``aprict.ramp_kernels``).

Each function returns the n (odd) taps h[k], k = -(n-1)/2 .. (n-1)/2, of a
filter applied by linear convolution, in float64 -- the reference notes that
float32 taps leave a visible DC error (src/aprict/ramp_kernels.py:38, :54):
  * ramp_kernel_ramlak: pi^2 (2 sinc(k) - sinc(k/2)^2) / dx, the band-limited
    ramp sampled at the pixel pitch (src/aprict/ramp_kernels.py:43-59);
    pi^2/dx at k = 0, -4/(k^2 dx) at odd k, 0 at even k != 0;
  * ramp_kernel: 8 / ((1 - 4 k^2) dx), the ramp with a sinc(f) pixel
    correction (:27-39);
  * hilbert_transform_kernel: 2/k, 0 at k = 0 (:62-77);
  * hilbert_transform_kernel_halfoffset: 2/(k + 1/2) (:80-94).
``apodize_hann`` multiplies a filter's response by the Hann window
(1 + cos 2 pi f)/2, f in cycles per pixel -- i.e. convolves the taps with
[1/4, 1/2, 1/4]. The reference has no apodisation; it is an addition.
"""

from __future__ import annotations

import numpy as np


def _k(n: int) -> np.ndarray:
    if n % 2 == 0:
        msg = "Window length must be odd."
        raise ValueError(msg)
    h = (n - 1) // 2
    return np.arange(-h, h + 1, dtype=np.float64)


def ramp_kernel(n: int, physpixsize: float | None = None) -> np.ndarray:
    """Ramp taps with the sinc(f) correction for a pixel of width physpixsize."""
    k = _k(n)
    return 8.0 / (1.0 - 4.0 * k * k) / (physpixsize or 1)


def ramp_kernel_ramlak(n: int, physpixsize: float | None = None) -> np.ndarray:
    """Ram-Lak taps, band-limited to the Nyquist frequency of pitch physpixsize."""
    k = _k(n)
    return np.pi**2 * (2.0 * np.sinc(k) - np.sinc(0.5 * k) ** 2) / (physpixsize or 1)


def hilbert_transform_kernel(n: int, physpixsize: float | None = None) -> np.ndarray:  # noqa: ARG001
    """Hilbert-transform taps 2/k (physpixsize has no effect)."""
    k = _k(n)
    out = np.zeros_like(k)
    nz = k != 0
    out[nz] = 2.0 / k[nz]
    return out


def hilbert_transform_kernel_halfoffset(n: int, physpixsize: float | None = None) -> np.ndarray:  # noqa: ARG001
    """Hilbert-transform taps 2/(k + 1/2) (physpixsize has no effect)."""
    k = _k(n)
    return 2.0 / (k + 0.5)


def apodize_hann(taps: np.ndarray) -> np.ndarray:
    """Taps of the filter multiplied in frequency by the Hann window (same length)."""
    return np.convolve(taps, np.array([0.25, 0.5, 0.25]), mode="same")


def odd_only(taps: np.ndarray, rtol: float = 1e-12) -> bool:
    """True if the taps at even nonzero offsets are zero to within rtol of the largest tap.

    The Ram-Lak formula evaluated with np.sinc leaves ~1e-16 relative residue
    at even offsets where the exact value is 0; dropping those taps changes a
    float32 result by far less than one ulp.
    """
    c = (len(taps) - 1) // 2
    even = np.concatenate([taps[c - 2 :: -2], taps[c + 2 :: 2]])
    return bool(even.size == 0 or np.max(np.abs(even)) <= rtol * np.max(np.abs(taps)))
