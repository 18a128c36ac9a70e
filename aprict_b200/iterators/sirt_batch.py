"""SIRT over many independent scans, two persistent launches per iteration.

Each scan is an ordinary :class:`~aprict_b200.iterators.SIRT_flatpanel`
(reference mode: x <- x + M (.) B (b - A x), src/aprict/iterators/sirt_vram.py:130-152),
set up exactly as on its own. :class:`SIRTBatch` then runs one iteration of
every scan as two launches -- the fused residuals r_i = b_i - A_i x_i of all
scans, then the backprojections x_i += M_i (.) B_i r_i of all scans -- through
:class:`~aprict_b200.batch.ScanBatch` plans, and ``iterate_graph(n)`` replays n
such iterations from one captured CUDA graph. Every scan ends with the same
iterate as running its own SIRT_flatpanel for the same number of iterations.
"""

from __future__ import annotations

from collections.abc import Sequence

import torch

from ..batch import ScanBatch
from ..cb import flatpanel as fp
from .sirt_vram import SIRT_flatpanel


class SIRTBatch:
    """Batched iterations of several reference-mode SIRT reconstructors."""

    def __init__(self, sirts: Sequence[SIRT_flatpanel]) -> None:
        if not sirts:
            msg = "SIRTBatch needs at least one SIRT_flatpanel"
            raise ValueError(msg)
        for s in sirts:
            if s._config.mode != "reference":  # noqa: SLF001
                msg = "SIRTBatch runs reference-mode SIRT only"
                raise NotImplementedError(msg)
        self._sirts = list(sirts)
        vols = [s.volume for s in sirts]
        scratch = [s._scratch for s in sirts]  # noqa: SLF001
        batch = ScanBatch(vols, scratch)
        self._fp = batch.plan_project(
            fp.ConfigProject(multiply_before_adding=-1), bases=[s._meas.data for s in sirts]  # noqa: SLF001
        )
        self._bp = batch.plan_backproject(
            [s._config_bp for s in sirts], multipliers=[s.preconditioner for s in sirts]  # noqa: SLF001
        )
        self._graph: torch.cuda.CUDAGraph | None = None
        self._graph_n = 0

    def __len__(self) -> int:
        return len(self._sirts)

    def _step(self) -> None:
        self._fp.run()
        self._bp.run()

    def _count(self, n: int) -> None:
        for s in self._sirts:
            s._iterations += n  # noqa: SLF001

    def iterate(self) -> None:
        """One iteration of every scan (two launches, asynchronous)."""
        self._step()
        self._count(1)

    def iterate_graph(self, n: int) -> None:
        """``n`` iterations of every scan replayed from one captured CUDA graph."""
        if n <= 0:
            return
        if self._graph is None or self._graph_n != n:
            # Planning loaded the kernels, so capture triggers no module load.
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                for _ in range(n):
                    self._step()
            self._graph, self._graph_n = g, n
        self._graph.replay()
        self._count(n)

    @property
    def sirts(self) -> list[SIRT_flatpanel]:
        """The per-scan reconstructors (volumes, preconditioners, counters)."""
        return list(self._sirts)
