"""A filter that does nothing (drop-in for ``aprict.cb.noop_filter.NoOpFilterer``,
src/aprict/cb/noop_filter.py): the same chunked interface as the ramp filters,
returning copies of the input, for pipelines that run unfiltered backprojection
through the same code path."""

from __future__ import annotations

import typing

import torch


class NoOpFilterer:
    """Copies projection chunks unchanged (one output per call, like a one-kernel filter)."""

    def __init__(self, *, proj_2d_shape: tuple[int, int], projs_per_batch: int = 2,
                 stream: torch.cuda.Stream | None = None) -> None:
        self.chunk_shape = (int(projs_per_batch), int(proj_2d_shape[0]), int(proj_2d_shape[1]))
        self.stream = stream

    @property
    def num_kerns(self) -> int:
        """The number of outputs per call."""
        return 1

    def filter_bulk_axis1_stream(self, arr: torch.Tensor, block: bool = True) -> typing.Iterator[tuple[list[torch.Tensor], torch.cuda.Event]]:
        """Generator of ([copy of the chunk], completion event) over chunks of ``projs_per_batch`` projections."""
        per = self.chunk_shape[0]
        for i in range(0, arr.shape[0], per):
            out = arr[i : i + per].clone()
            ev = torch.cuda.Event()
            ev.record()
            if block:
                ev.synchronize()
            yield [out], ev

    def filter_bulk_axis1_concat(self, arr: torch.Tensor, block: bool = True) -> tuple[list[torch.Tensor], torch.cuda.Event]:
        """([copy of the whole array], completion event)."""
        out = arr.clone()
        ev = torch.cuda.Event()
        ev.record()
        if block:
            ev.synchronize()
        return [out], ev
