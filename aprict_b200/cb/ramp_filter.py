"""Ramp filtering with cosine weighting (drop-in for ``aprict.cb.FBPFilterer`` / ``RampFilterer``).

The reference filters a chunk of projections by zero-padding every detector
row to next_fast_len(2 nu - 1), running cuFFT R2C, multiplying by the tap
spectrum (complex128) and C2R (src/aprict/cb/ramp_filter.py:83-240), after a
cosine weight per pixel (:407-449, applied at :685-689). That is a linear
convolution, evaluated here in one launch for the whole projection stack with
the weights fused into the staging of each row: by a shared-memory FFT
(``aprict_b200_ramp_filter_fft``, from tables built once per filter) for rows
of 128 to 2048 samples, else directly (``aprict_b200_ramp_filter``).

``FBPFilterer`` also filters along tilted lines for the cone-cylinder FBP
(:577-886): each projection is padded to a wider frame, rotated by a random
(or forced) angle, weighted, letterboxed, ramp-filtered along u and rotated
back. Here the padding, rotation, weights and letterbox of a stack are one
``aprict_b200_rotate_projections`` launch, the filter one convolution launch
per kernel, and the back-rotation and crop one more launch per kernel.
"""

from __future__ import annotations

import enum
import math
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
            self._taps.append(_lib.upload(h.astype(np.float32)))
        # Rows of 128 to 2048 samples are filtered by FFT from tables (kernel
        # spectrum and twiddles) built here once per filter, as the reference
        # keeps each filter's spectrum (ramp_filter.py:83-137); other lengths by
        # the direct convolution of the taps.
        lib = _lib.lib()
        nbytes = int(lib.aprict_b200_ramp_fft_tables_bytes(nu))
        self._fft_tables: list[torch.Tensor | None] = []
        for t in self._taps:
            tab = None
            if nbytes > 0:
                tab = torch.empty(nbytes, dtype=torch.uint8, device=t.device)
                _lib.check(lib.aprict_b200_ramp_fft_tables(t.data_ptr(), nu, tab.data_ptr(), _stream()), "ramp_fft_tables")
            self._fft_tables.append(tab)
        self._tables_ready = torch.cuda.Event()
        self._tables_ready.record()

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
        lib = _lib.lib()
        torch.cuda.current_stream().wait_event(self._tables_ready)
        for taps, odd, tab, out in zip(self._taps, self._odd, self._fft_tables, outs):
            dout = _desc(out)
            if tab is not None:
                _lib.check(
                    lib.aprict_b200_ramp_filter_fft(
                        _lib.ptr(din), data.data_ptr(), _lib.ptr(dout), out.data_ptr(), tab.data_ptr(),
                        wptr, wsu, wsv, float(scale), _stream(),
                    ),
                    "ramp_filter_fft",
                )
            else:
                _lib.check(
                    lib.aprict_b200_ramp_filter(
                        _lib.ptr(din), data.data_ptr(), _lib.ptr(dout), out.data_ptr(), taps.data_ptr(), int(odd),
                        wptr, wsu, wsv, float(scale), _stream(),
                    ),
                    "ramp_filter",
                )
        return outs

    def filter_bulk_axis1_stream(self, arr: torch.Tensor, block: bool = True):  # noqa: ANN201
        """Generator of (filtered chunks, one per filter; completion event) over chunks of
        ``projs_per_batch`` projections (ramp_filter.py:242-259)."""
        per = self.chunk_shape[0]
        for i in range(0, arr.shape[0], per):
            outs = self.filter(arr[i : i + per])
            ev = torch.cuda.Event()
            ev.record()
            if block:
                ev.synchronize()
            yield outs, ev

    def filter_bulk_axis1_concat(self, arr: torch.Tensor, block: bool = True) -> tuple[list[torch.Tensor], torch.cuda.Event]:
        """All projections filtered at once: (one (M, nu, nv) array per filter, completion event)
        (ramp_filter.py:261-305; the convolution kernel takes any number of views per launch)."""
        outs = self.filter(arr)
        ev = torch.cuda.Event()
        ev.record()
        if block:
            ev.synchronize()
        return outs, ev


def frame_weight_mask(frame_shape: tuple[int, int], physpixwid: float, L: float, fdk: bool) -> np.ndarray:  # noqa: N803
    """FP64 weights over the padded frame, computed from the reference's float32
    pixel grids (ramp_filter.py:407-449): 1 / sqrt(1 + u^2 + v^2) for FDK,
    otherwise 1 / ((1 + v^2)^(3/2) sqrt(1 + u^2 + v^2)), u and v in units of L."""
    nu_e, nv_e = int(frame_shape[0]), int(frame_shape[1])
    uarr = physpixwid / L * (np.arange(nu_e, dtype=np.float32) - (nu_e - 1) / 2)
    varr = physpixwid / L * (np.arange(nv_e, dtype=np.float32) - (nv_e - 1) / 2)
    if fdk:
        mask = 1 / np.sqrt(1 + np.square(varr[np.newaxis, :]) + np.square(uarr[:, np.newaxis]))
    else:
        mask = 1 / (np.float_power(np.sqrt(1 + np.square(varr[np.newaxis, :])), 3)
                    * np.sqrt(1 + np.square(varr[np.newaxis, :]) + np.square(uarr[:, np.newaxis])))
    return np.ascontiguousarray(mask, dtype=np.float64)


class FBPFilterer:
    """Weighted ramp (and optionally Hilbert) filtering for FBP (ramp_filter.py:333-886).

    Fan-beam and FDK modes (``_hacky_fan_beam_mode`` / ``_hacky_fdk_mode``)
    at rotation angle 0 fold the weights into the convolution's staging.
    Otherwise each projection is filtered along lines tilted by its rotation
    angle (random uniform in [-zeta, zeta], one ``rng.random()`` per
    projection, or ``force_rotation_angle``).
    """

    class SamplingStrategy(enum.Enum):
        """Rotation sampling strategies of the reference."""

        SINGLE_ROTATION_RANDOM_UNIFORM = 1

    # scratch budget of the tilted path per sub-chunk of views
    _SCRATCH_BYTES = 512 << 20

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
        self.projs_per_batch = int(projs_per_batch)
        self.rng = np.random.default_rng(seed=None) if rng is None else rng
        self._include_hilbert_transform = include_hilbert_transform_in_output
        self._max_abs_rotation_angle = self.get_max_abs_rotation_angle(self.proj_2d_shape, physpixwid, L)
        if limit_zeta is not None:
            self._max_abs_rotation_angle = min(self._max_abs_rotation_angle, limit_zeta)
        self._expanded_2d_shape = self.get_expanded_proj_2d_shape(
            self.proj_2d_shape, self._max_abs_rotation_angle, _hacky_fan_beam_mode, _hacky_fdk_mode
        )
        self.chunk_shape = (self.projs_per_batch, *self._expanded_2d_shape)
        funcs: tuple[KernFunc, ...] = (ramp_kernels.ramp_kernel_ramlak,)
        if include_hilbert_transform_in_output:
            funcs += (ramp_kernels.hilbert_transform_kernel,)
        # taps use the pixel pitch projected to distance 1 from the source (:393-395)
        self.rfilt = RampFilterer(
            physpixwid=physpixwid / L,
            proj_2d_shape=self._expanded_2d_shape,
            projs_per_batch=projs_per_batch,
            override_kern_funcs=funcs,
            apodization=apodization,
        )
        self._mask_host = frame_weight_mask(self._expanded_2d_shape, physpixwid, L, _hacky_fdk_mode)
        self._mask = _lib.upload(self._mask_host)
        # Angle-0 fan/FDK path: the same weights folded into the convolution (FP32).
        nu, nv = self.proj_2d_shape
        u = physpixwid / L * (np.arange(nu, dtype=np.float64) - (nu - 1) / 2)
        v = physpixwid / L * (np.arange(nv, dtype=np.float64) - (nv - 1) / 2)
        uu, vv = u[:, None], v[None, :]
        if _hacky_fdk_mode:
            w = 1.0 / np.sqrt(1 + vv**2 + uu**2)
        else:
            w = 1.0 / (np.sqrt(1 + vv**2) ** 3 * np.sqrt(1 + vv**2 + uu**2))
        self._weights_host = w
        self._weights = _lib.upload(w.astype(np.float32))

    # ---- the reference's helpers (ramp_filter.py:439-562) ----

    def advance_rng(self, amount: int) -> None:
        """Advance the internal rng by ``amount`` draws (as if that many projections were filtered)."""
        for _ in range(amount):
            self.rng.random()

    def uniform_rng(self, low: float, high: float, len: int) -> np.ndarray:  # noqa: A002
        """``len`` angles ``low + (high - low) * rng.random()`` as float32, one draw each (:443-460)."""
        out = np.empty((len,), dtype=np.float32)
        for i in range(len):
            out[i] = low + (high - low) * self.rng.random()
        return out

    def get_letterbox_slice(self, rotation_angle: float) -> slice:
        """Fractional column range of the rotated detector's vertical extent (:462-492)."""
        if abs(rotation_angle) > self._max_abs_rotation_angle:
            msg = "Invalid rotation angle entered."
            raise ValueError(msg)
        mid_index = (self._expanded_2d_shape[1] - 1) / 2
        disc = self.L / self.physpixwid * np.sqrt(
            np.maximum(np.square(np.cos(rotation_angle) / np.cos(self._max_abs_rotation_angle)) - 1, 0)
        )
        return slice(mid_index - disc, mid_index + disc)

    def _letterbox_columns(self, rotation_angle: float) -> np.ndarray:
        """Per-column factors of the letterbox multiplies (:690-749)."""
        sl = self.get_letterbox_slice(rotation_angle)
        w = np.ones(self._expanded_2d_shape[1])
        i1, i2 = round(sl.start), round(sl.stop)
        if i1 == i2:
            w[i1] = sl.stop - sl.start
            w[:i1] = 0
            w[i1 + 1 :] = 0
        else:
            w[i1] = (i1 + 1 / 2) - sl.start
            w[i2] = sl.stop - (i2 - 1 / 2)
            w[:i1] = 0
            w[i2 + 1 :] = 0
        return w

    @property
    def zeta(self) -> float:
        """The largest rotation angle this object accommodates."""
        return self._max_abs_rotation_angle

    @classmethod
    def get_max_abs_rotation_angle(cls, proj_2d_shape: tuple[int, int], physpixwid: float, L: float) -> float:  # noqa: N803
        """Half the vertical cone angle (ramp_filter.py:494-514)."""
        nu, nv = int(proj_2d_shape[0]), int(proj_2d_shape[1])
        return float(np.arctan2(nv * physpixwid / 2, np.sqrt(L**2 + (nu * physpixwid / 2) ** 2)))

    @classmethod
    def get_expanded_proj_2d_shape(
        cls,
        proj_2d_shape: tuple[int, int],
        max_abs_rotation_angle: float,
        _hacky_fan_beam_mode: bool = False,
        _hacky_fdk_mode: bool = False,
    ) -> tuple[int, int]:
        """The padded frame that holds every rotated projection (:516-562)."""
        if _hacky_fan_beam_mode and _hacky_fdk_mode:
            msg = "Cannot use both _hacky_fan_beam_mode and _hacky_fdk_mode."
            raise ValueError(msg)
        nu, nv = int(proj_2d_shape[0]), int(proj_2d_shape[1])
        if _hacky_fan_beam_mode or _hacky_fdk_mode:
            return nu, nv
        s, c = np.sin(max_abs_rotation_angle), np.cos(max_abs_rotation_angle)
        w, h = int(np.ceil(nv * s + nu * c)), int(np.ceil(nv))
        return w + (w - nu) % 2, h + (h - nv) % 2

    @property
    def weights(self) -> np.ndarray:
        """The (nu, nv) weights of the angle-0 fan/FDK path (float64)."""
        return self._weights_host.copy()

    @property
    def mask(self) -> np.ndarray:
        """The weight mask over the padded frame (float64)."""
        return self._mask_host.copy()

    # ---- filtering ----

    def _angles(self, n: int, force_rotation_angle: float | None) -> np.ndarray:
        if force_rotation_angle is None:
            return self.uniform_rng(-self._max_abs_rotation_angle, self._max_abs_rotation_angle, n)
        return force_rotation_angle * np.ones((n,), dtype=np.float32)

    def _letterbox_matrix(self, angles: np.ndarray) -> np.ndarray:
        """``_letterbox_columns`` of every angle at once, (len(angles), nv_e): the same
        arithmetic elementwise, without a Python loop over the views."""
        ang = np.asarray(angles)
        if np.any(np.abs(ang) > self._max_abs_rotation_angle):
            msg = "Invalid rotation angle entered."
            raise ValueError(msg)
        nv_e = self._expanded_2d_shape[1]
        mid_index = (nv_e - 1) / 2
        disc = self.L / self.physpixwid * np.sqrt(
            np.maximum(np.square(np.cos(ang) / np.cos(self._max_abs_rotation_angle)) - 1, 0)
        )
        start, stop = mid_index - disc, mid_index + disc
        i1, i2 = np.round(start).astype(np.int64), np.round(stop).astype(np.int64)
        cols = np.arange(nv_e)[None, :]
        w = ((cols >= i1[:, None]) & (cols <= i2[:, None])).astype(np.float64)
        rows = np.arange(len(ang))
        same = i1 == i2
        w[rows, i1] = np.where(same, stop - start, (i1 + 1 / 2) - start)
        w[rows[~same], i2[~same]] = (stop - (i2 - 1 / 2))[~same]
        return w

    @staticmethod
    def _cs(angles_deg: np.ndarray) -> np.ndarray:
        # the library's chain: numpy.deg2rad in the angles' dtype, then math.cos / math.sin
        rad = np.deg2rad(angles_deg)
        return np.array([[math.cos(r), math.sin(r)] for r in rad], dtype=np.float64)

    def _filter_tilted(self, data: torch.Tensor, angles: np.ndarray, outs: list[torch.Tensor]) -> None:
        """Filter (n, nu, nv) ``data`` along lines tilted by ``angles`` into ``outs``."""
        n = data.shape[0]
        nu_e, nv_e = self._expanded_2d_shape
        nu, nv = self.proj_2d_shape
        padx, pady = (nu_e - nu) // 2, (nv_e - nv) // 2
        cu, cv = (nu_e - 1) / 2, (nv_e - 1) / 2
        hacky = self.hacky_fan_beam_mode or self.hacky_fdk_mode
        per = max(1, min(n, self._SCRATCH_BYTES // (4 * nu_e * nv_e * (1 + self.rfilt.num_kerns))))
        lib = _lib.lib()
        for a in range(0, n, per):
            b = min(n, a + per)
            ang = angles[a:b]
            cs_fwd = _lib.upload(self._cs(-180 / np.pi * ang))
            cs_bwd = _lib.upload(self._cs(180 / np.pi * ang))
            colw = None
            if not hacky:
                colw = _lib.upload(self._letterbox_matrix(ang))
            frame = torch.empty((b - a, nu_e, nv_e), dtype=torch.float32, device=data.device)
            src = data[a:b]
            d_src, d_frame = _desc(src), _desc(frame)  # kept alive across the calls
            _lib.check(
                lib.aprict_b200_rotate_projections(
                    _lib.ptr(d_src), src.data_ptr(), _lib.ptr(d_frame), frame.data_ptr(), cs_fwd.data_ptr(),
                    cu, cv, padx, pady, 0, 0, self._mask.data_ptr(), None if colw is None else colw.data_ptr(),
                    _stream(),
                ),
                "rotate_projections",
            )
            filtered = self.rfilt.filter(frame)
            for f, out in zip(filtered, outs):
                dst = out[a:b]
                d_f, d_dst = _desc(f), _desc(dst)
                _lib.check(
                    lib.aprict_b200_rotate_projections(
                        _lib.ptr(d_f), f.data_ptr(), _lib.ptr(d_dst), dst.data_ptr(), cs_bwd.data_ptr(),
                        cu, cv, 0, 0, padx, pady, None, None, _stream(),
                    ),
                    "rotate_projections",
                )

    def filter_bulk_axis1_concat(
        self,
        arr: torch.Tensor | np.ndarray,
        clear_gpu_cache_regularly: bool = True,  # noqa: ARG002
        force_rotation_angle: float | None = None,
        block: bool = True,
    ) -> tuple[list[torch.Tensor], torch.cuda.Event]:
        """Filter a whole (M, nu, nv) stack; returns (one (M, nu, nv) array per filter, completion event)."""
        if tuple(arr.shape[1:]) != self.proj_2d_shape:
            msg = "Wrong input size."
            raise ValueError(msg)
        if isinstance(arr, np.ndarray):
            data = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32)).cuda()
        else:
            data = arr
            if data.dtype != torch.float32 or not data.is_cuda:
                msg = "arr must be a float32 CUDA tensor or a host array"
                raise ValueError(msg)
        n = data.shape[0]
        angles = self._angles(n, force_rotation_angle)
        hacky = self.hacky_fan_beam_mode or self.hacky_fdk_mode
        if hacky and not np.any(angles):
            outs = self.rfilt.filter(data, weights=self._weights)  # padded frame == detector: no resampling
        else:
            outs = [torch.empty((n, *self.proj_2d_shape), dtype=torch.float32, device=data.device)
                    for _ in range(self.rfilt.num_kerns)]
            self._filter_tilted(data, angles, outs)
        ev = torch.cuda.Event()
        ev.record()
        if block:
            ev.synchronize()
        return outs, ev

    def filter_bulk_axis1_stream(self, arr: torch.Tensor | np.ndarray, block: bool = True, clear_gpu_cache_regularly: bool = False,
                                 force_rotation_angle: float | None = None):  # noqa: ANN201
        """Generator form: yields (filtered arrays, event) per chunk of projs_per_batch projections."""
        if tuple(arr.shape[1:]) != self.proj_2d_shape:
            msg = "Wrong input size."
            raise ValueError(msg)
        for i in range(0, arr.shape[0], self.projs_per_batch):
            yield self.filter_bulk_axis1_concat(arr[i : i + self.projs_per_batch], clear_gpu_cache_regularly,
                                                force_rotation_angle, block)
