"""Many independent scans in one persistent launch per operation.

The reference projects and backprojects one scan per call
(src/aprict/cb/flatpanel.py:997-1281): a workload of many small, uneven scans
(different volume sizes, view counts and detectors) then runs as a long
sequence of launches, each too small to fill the GPU, with a host
synchronisation per scan. :class:`ScanBatch` instead plans all scans of a
batch at once (``aprict_b200_batch_plan``) and runs each operation as one
persistent launch (``aprict_b200_batch_run``) whose CTAs pull detector tiles
or volume bricks of every scan from a shared counter. Each scan's result is
the one its one-scan call (:func:`~aprict_b200.cb.flatpanel.project`,
:func:`~aprict_b200.cb.flatpanel.backproject`) gives.

A :class:`BatchPlan` records the device buffers it was built for; it can be
run any number of times (and captured in a CUDA graph) while they live.
"""

from __future__ import annotations

from collections.abc import Sequence

import numpy as np
import torch

from . import _lib
from . import _structs as S
from .cb import flatpanel as fp
from .volume import Volume

PROJECT, BACKPROJECT = 0, 1


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class BatchPlan:
    """A planned batch operation: the host image and its device copy."""

    def __init__(self, op: int, scans: np.ndarray, configs: np.ndarray, keepalive: list) -> None:
        lib = _lib.lib()
        n = int(scans.shape[0])
        nbytes = int(lib.aprict_b200_batch_plan_bytes(op, n))
        if nbytes == 0:
            msg = "empty batch"
            raise ValueError(msg)
        raw = np.zeros(nbytes + 256, np.uint8)
        off = (-raw.ctypes.data) % 256
        self._host = raw[off : off + nbytes]
        _lib.check(
            lib.aprict_b200_batch_plan(op, _lib.ptr(scans), n, _lib.ptr(configs), self._host.ctypes.data, nbytes),
            "batch_plan",
        )
        self._dev = _lib.upload(self._host)
        if self._dev.data_ptr() % 256:
            msg = "device plan is not 256-byte aligned"
            raise RuntimeError(msg)
        self._keep = keepalive  # the buffers whose addresses the plan holds
        self.op = op
        self.n_scans = n

    def run(self, block: bool = False) -> None:
        """Enqueue the operation on the current stream."""
        _lib.check(_lib.lib().aprict_b200_batch_run(self._host.ctypes.data, self._dev.data_ptr(), _stream()), "batch_run")
        if block:
            torch.cuda.current_stream().synchronize()


def _packed(items: list[np.ndarray], dtype: np.dtype) -> np.ndarray:
    """An array of C structs with the exact C layout (np.stack would drop padding)."""
    out = np.zeros(len(items), dtype)
    for i, it in enumerate(items):
        out[i] = it
    return out


def _scan_record(volume: Volume, projs: fp.ProjectionSet) -> np.ndarray:
    if projs.data is None:
        msg = "every ProjectionSet of a batch needs a data buffer"
        raise ValueError(msg)
    if projs.proj_specs.ndim != 1:
        msg = "batched scans take one-dimensional view lists"
        raise NotImplementedError(msg)
    if not volume.data.is_cuda:
        msg = "Volume data must live on the GPU."
        raise ValueError(msg)
    if volume.data.dtype != torch.float32 or projs.data.dtype != torch.float32:
        msg = "batched scans take float32 volumes and projections (one-scan calls take float16 / float64 too)"
        raise NotImplementedError(msg)
    rec = np.zeros((), S.scan)
    d = projs.data
    rec["specs_dev"] = projs.specs_device().data_ptr()
    rec["projs"] = _lib.proj_desc(tuple(d.shape), tuple(d.stride()))
    rec["projs_dev"] = d.data_ptr()
    rec["vol"] = volume._desc()  # noqa: SLF001
    rec["vol_dev"] = volume.data.data_ptr()
    return rec


class ScanBatch:
    """Independent scans ``(volumes[i], projs[i])`` processed together."""

    def __init__(self, volumes: Sequence[Volume], projs: Sequence[fp.ProjectionSet]) -> None:
        if len(volumes) != len(projs) or not volumes:
            msg = "a batch needs one ProjectionSet per volume and at least one scan"
            raise ValueError(msg)
        for p in projs:
            p.create_buffer(dtype=np.float32, existing_ok=True)
        self.volumes = list(volumes)
        self.projs = list(projs)

    def __len__(self) -> int:
        return len(self.volumes)

    def _records(self) -> np.ndarray:
        return _packed([_scan_record(v, p) for v, p in zip(self.volumes, self.projs, strict=True)], S.scan)

    @staticmethod
    def _per_scan(cfg, n: int) -> list:
        if isinstance(cfg, Sequence):
            if len(cfg) != n:
                msg = f"{len(cfg)} configs for {n} scans"
                raise ValueError(msg)
            return list(cfg)
        return [cfg] * n

    def plan_project(
        self,
        configs: fp.ConfigProject | Sequence[fp.ConfigProject] | None = None,
        *,
        bases: Sequence[torch.Tensor] | None = None,
    ) -> BatchPlan:
        """Plan ``projs[i] += mba A volumes[i]``, or with ``bases`` the fused
        ``projs[i] = bases[i] + mba A volumes[i]`` (see ``project_residual``)."""
        n = len(self)
        cfgs = self._per_scan(configs if configs is not None else fp.ConfigProject(), n)
        recs = self._records()
        keep: list = [*self.volumes, *self.projs]
        if bases is not None:
            if len(bases) != n:
                msg = f"{len(bases)} bases for {n} scans"
                raise ValueError(msg)
            for i, b in enumerate(bases):
                d = self.projs[i].data
                if tuple(b.shape) != tuple(d.shape) or b.stride() != d.stride() or not b.is_cuda or b.dtype != torch.float32:
                    msg = "each base must be a float32 CUDA tensor with the shape and strides of its projection data"
                    raise ValueError(msg)
                recs[i]["base_dev"] = b.data_ptr()
            keep += list(bases)
        conf = _packed([c.contents for c in cfgs], S.project_config)
        return BatchPlan(PROJECT, recs, conf, keep)

    def plan_backproject(
        self,
        configs: fp.ConfigBackproject | Sequence[fp.ConfigBackproject],
        *,
        multipliers: Sequence[Volume | None] | None = None,
    ) -> BatchPlan:
        """Plan ``volumes[i] += multipliers[i] (.) BP projs[i]`` with the same
        checks as :func:`~aprict_b200.cb.flatpanel.backproject`."""
        n = len(self)
        cfgs = self._per_scan(configs, n)
        mults = list(multipliers) if multipliers is not None else [None] * n
        if len(mults) != n:
            msg = f"{len(mults)} multipliers for {n} scans"
            raise ValueError(msg)
        recs = self._records()
        keep: list = [*self.volumes, *self.projs]
        for i, (c, m) in enumerate(zip(cfgs, mults, strict=True)):
            v = self.volumes[i]
            if bool(c.contents["apply_summand_multiplier"]) != (m is not None):
                msg = "To prevent unintended behaviour, the config 'apply_summand_multiplier' must be true if and only if a summand_multiplier is included."
                raise ValueError(msg)
            if m is not None:
                if m.shape != v.shape or m.order != v.order or m.dtype != v.dtype:
                    msg = "each multiplier must match its volume's shape, dtype and order"
                    raise ValueError(msg)
                recs[i]["multiplier_dev"] = m.data.data_ptr()
                keep.append(m)
            if int(c.contents["weighting_preset"]) > 6:
                msg = "Backprojection weighting preset 7 (the GBC formula) is not implemented."
                raise NotImplementedError(msg)
        conf = _packed([c.contents for c in cfgs], S.backproject_config)
        return BatchPlan(BACKPROJECT, recs, conf, keep)

    def project(self, configs=None, *, bases=None, block: bool = False) -> None:
        """Plan and run one batched projection."""
        self.plan_project(configs, bases=bases).run(block=block)

    def backproject(self, configs, *, multipliers=None, block: bool = False) -> None:
        """Plan and run one batched backprojection."""
        self.plan_backproject(configs, multipliers=multipliers).run(block=block)


__all__ = ["BACKPROJECT", "PROJECT", "BatchPlan", "ScanBatch"]
