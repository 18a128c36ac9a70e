"""Ramp filtering with cosine weighting (drop-in for ``aprict.cb.FBPFilterer`` / ``RampFilterer``).

The reference filters a chunk of projections by zero-padding every detector
row to next_fast_len(2 nu - 1), running cuFFT R2C, multiplying by the tap
spectrum (complex128) and C2R (src/aprict/cb/ramp_filter.py:83-240), after a
cosine weight per pixel (:407-449, applied at :685-689). That is a linear
convolution, evaluated here directly by ``aprict_b200_ramp_filter`` (a
shared-memory convolution kernel), one launch for the whole projection stack
with the weights fused into the staging of each row.

Scope: the fan-beam and FDK modes (``_hacky_fan_beam_mode`` /
``_hacky_fdk_mode``), i.e. rotation angle 0. The cone-cylinder path that
rotates each projection before filtering (:577-886) is not implemented and
raises NotImplementedError.
"""

from __future__ import annotations

import enum
import typing

import numpy as np
import torch

from .. import _lib, ramp_kernels

KernFunc = typing.Callable[[int, float | None], np.ndarray]


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _desc(t: torch.Tensor) -> np.ndarray:
    return _lib.proj_desc(tuple(t.shape[-3:]), tuple(t.stride()[-3:]))


class RampFilterer:
    """Linear convolution of every detector row (axis 1 of (M, nu, nv)) with 1-D taps."""

    def __init__(
        self,
        *,
        physpixwid: float = 1,
        proj_2d_shape: tuple[int, int],
        projs_per_batch: int = 2,
        stream: torch.cuda.Stream | None = None,
        override_kern_funcs: tuple[KernFunc, ...] | None = None,
        apodization: str | None = None,
    ) -> None:
        self.chunk_shape = (int(projs_per_batch), int(proj_2d_shape[0]), int(proj_2d_shape[1]))
        self.physpixwid = float(physpixwid)
        self.stream = stream
        funcs = override_kern_funcs or (ramp_kernels.ramp_kernel_ramlak,)
        nu = self.chunk_shape[1]
        self._taps_host: list[np.ndarray] = []
        self._taps: list[torch.Tensor] = []
        self._odd: list[bool] = []
        for f in funcs:
            h = np.asarray(f(2 * nu - 1, self.physpixwid), dtype=np.float64)
            if apodization == "hann":
                h = ramp_kernels.apodize_hann(h)
            elif apodization is not None:
                msg = f"unknown apodization {apodization!r}"
                raise ValueError(msg)
            self._taps_host.append(h)
            self._odd.append(ramp_kernels.odd_only(h))
            self._taps.append(torch.from_numpy(h.astype(np.float32)).cuda())

    @property
    def num_kerns(self) -> int:
        """How many filters are applied (outputs per call)."""
        return len(self._taps)

    @property
    def taps(self) -> list[np.ndarray]:
        """The float64 taps h[-(nu-1)] .. h[nu-1] of each filter."""
        return [h.copy() for h in self._taps_host]

    def filter(
        self,
        data: torch.Tensor,
        *,
        weights: torch.Tensor | None = None,
        scale: float = 1.0,
        outs: list[torch.Tensor] | None = None,
    ) -> list[torch.Tensor]:
        """Filter (M, nu, nv) data along nu; returns one (M, nu, nv) tensor per filter."""
        if data.dim() != 3 or data.shape[1] != self.chunk_shape[1] or data.shape[2] != self.chunk_shape[2]:
            msg = "Input projection array shape does not match the shape initialised for this filtering object."
            raise ValueError(msg)
        if data.dtype != torch.float32 or not data.is_cuda:
            msg = "data must be a float32 CUDA tensor"
            raise ValueError(msg)
        if outs is None:
            outs = [torch.empty_like(data) for _ in self._taps]
        wptr, wsu, wsv = None, 0, 0
        if weights is not None:
            if tuple(weights.shape) != tuple(data.shape[1:]) or weights.dtype != torch.float32:
                msg = "weights must be a float32 (nu, nv) tensor"
                raise ValueError(msg)
            wptr, (wsu, wsv) = weights.data_ptr(), weights.stride()
        din = _desc(data)
        for taps, odd, out in zip(self._taps, self._odd, outs):
            dout = _desc(out)
            _lib.check(
                _lib.lib().aprict_b200_ramp_filter(
                    _lib.ptr(din), data.data_ptr(), _lib.ptr(dout), out.data_ptr(), taps.data_ptr(), int(odd),
                    wptr, wsu, wsv, float(scale), _stream(),
                ),
                "ramp_filter",
            )
        return outs


class FBPFilterer:
    """Cosine-weighted ramp (and optionally Hilbert) filtering for FBP (ramp_filter.py:333-940)."""

    class SamplingStrategy(enum.Enum):
        """Rotation sampling strategies of the reference (only angle 0 is implemented)."""

        SINGLE_ROTATION_RANDOM_UNIFORM = 1

    def __init__(
        self,
        *,
        L: float,  # noqa: N803
        physpixwid: float,
        proj_2d_shape: tuple[int, int],
        projs_per_batch: int = 3,
        sampling_strategy: SamplingStrategy = SamplingStrategy.SINGLE_ROTATION_RANDOM_UNIFORM,
        limit_zeta: float | None = None,
        include_hilbert_transform_in_output: bool = False,
        _hacky_fan_beam_mode: bool = False,
        _hacky_fdk_mode: bool = False,
        rng: np.random.Generator | None = None,
        apodization: str | None = None,
    ) -> None:
        if _hacky_fan_beam_mode and _hacky_fdk_mode:
            msg = "Cannot use both _hacky_fan_beam_mode and _hacky_fdk_mode."
            raise ValueError(msg)
        self.L = float(L)
        self.physpixwid = float(physpixwid)
        self.proj_2d_shape = (int(proj_2d_shape[0]), int(proj_2d_shape[1]))
        self.hacky_fan_beam_mode = _hacky_fan_beam_mode
        self.hacky_fdk_mode = _hacky_fdk_mode
        self.ss = sampling_strategy
        self.rng = np.random.default_rng() if rng is None else rng
        self._max_abs_rotation_angle = self.get_max_abs_rotation_angle(self.proj_2d_shape, physpixwid, L)
        if limit_zeta is not None:
            self._max_abs_rotation_angle = min(self._max_abs_rotation_angle, limit_zeta)
        funcs: tuple[KernFunc, ...] = (ramp_kernels.ramp_kernel_ramlak,)
        if include_hilbert_transform_in_output:
            funcs += (ramp_kernels.hilbert_transform_kernel,)
        # taps use the pixel pitch projected to distance 1 from the source (:393-395)
        self.rfilt = RampFilterer(
            physpixwid=physpixwid / L,
            proj_2d_shape=self.proj_2d_shape,
            projs_per_batch=projs_per_batch,
            override_kern_funcs=funcs,
            apodization=apodization,
        )
        nu, nv = self.proj_2d_shape
        u = physpixwid / L * (np.arange(nu, dtype=np.float64) - (nu - 1) / 2)
        v = physpixwid / L * (np.arange(nv, dtype=np.float64) - (nv - 1) / 2)
        uu, vv = u[:, None], v[None, :]
        if _hacky_fdk_mode:
            w = 1.0 / np.sqrt(1 + vv**2 + uu**2)
        else:
            w = 1.0 / (np.sqrt(1 + vv**2) ** 3 * np.sqrt(1 + vv**2 + uu**2))
        self._weights_host = w
        self._weights = torch.from_numpy(w.astype(np.float32)).cuda()

    @property
    def zeta(self) -> float:
        """Largest rotation angle the reference's rotated filtering would accept."""
        return self._max_abs_rotation_angle

    @classmethod
    def get_max_abs_rotation_angle(cls, proj_2d_shape: tuple[int, int], physpixwid: float, L: float) -> float:  # noqa: N803
        """Half the vertical cone angle (ramp_filter.py:494-514)."""
        nu, nv = int(proj_2d_shape[0]), int(proj_2d_shape[1])
        return float(np.arctan2(nv * physpixwid / 2, np.sqrt(L**2 + (nu * physpixwid / 2) ** 2)))

    @property
    def weights(self) -> np.ndarray:
        """The (nu, nv) cosine weights (float64)."""
        return self._weights_host.copy()

    def filter_bulk_axis1_concat(
        self,
        arr: torch.Tensor | np.ndarray,
        block: bool = True,
        clear_gpu_cache_regularly: bool = False,  # noqa: ARG002
        force_rotation_angle: float | None = None,
    ) -> tuple[list[torch.Tensor], torch.cuda.Event]:
        """Weight and filter a whole (M, nu, nv) stack; returns (filtered arrays, completion event)."""
        if not (self.hacky_fan_beam_mode or self.hacky_fdk_mode) or (force_rotation_angle not in (None, 0, 0.0)):
            msg = "Only the fan-beam and FDK filtering modes (rotation angle 0) are implemented."
            raise NotImplementedError(msg)
        data = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32)).cuda() if isinstance(arr, np.ndarray) else arr
        if tuple(data.shape[1:]) != self.proj_2d_shape:
            msg = "Wrong input size."
            raise ValueError(msg)
        outs = self.rfilt.filter(data, weights=self._weights)
        ev = torch.cuda.Event()
        ev.record()
        if block:
            ev.synchronize()
        return outs, ev

    def filter_bulk_axis1_stream(self, arr: torch.Tensor | np.ndarray, block: bool = True, **kw: object):  # noqa: ANN201
        """Generator form: yields (filtered arrays, event) per chunk of projs_per_batch projections."""
        n = arr.shape[0]
        per = self.rfilt.chunk_shape[0]
        for i in range(0, n, per):
            yield self.filter_bulk_axis1_concat(arr[i : i + per], block=block, **kw)
