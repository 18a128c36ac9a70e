"""SIRT on the GPU (drop-in for ``aprict.iterators.SIRT_flatpanel``).

The reference's "SIRT" (src/aprict/iterators/sirt_vram.py:31-157) is a
Jacobi-preconditioned Landweber iteration

    x <- x + M (.) B (b - A x),     M ~ 1 / diag(B A 1)

with A the exact Siddon projector, B the (by default fast) backprojector with
a cylinder mask and a detector-edge taper, and M built once in ``__init__``
(:83-118). That is reproduced operation for operation (``mode="reference"``).

Per iteration the reference runs a copy, one projection launch, ceil(M/10)
backprojection launches and two host synchronisations (:130-152). Here an
iteration is two kernels -- the fused residual r = b - A x
(``project_residual``) and one all-view backprojection that applies M and
updates x in its epilogue -- and ``iterate_graph(n)`` replays n iterations as
one captured CUDA graph with no host synchronisation.

``mode="classical"`` runs textbook SIRT, x <- x + C B R (b - A x) with
R = 1/(A 1) and C = 1/(B 1), B the exact (matched) backprojector.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import torch

from .. import Volume
from ..cb import flatpanel as fp


@dataclasses.dataclass(frozen=True, kw_only=True)
class _Config:
    """Configuration of the SIRT iterator (sirt_vram.py:45-55)."""

    fast_backproject: bool = True
    soft_from_cylinder_relrad: float | None = 0.95
    bp_soft_from_detedge_relrad: float | None = 0.95
    mode: str = "reference"  # "reference" | "classical"


class _HostPipeline:
    """Buffers, streams and events of SIRT_flatpanel.iterate_from_host."""

    def __init__(self, meas: torch.Tensor, vol: torch.Tensor) -> None:
        self.up, self.down = torch.cuda.Stream(), torch.cuda.Stream()
        self.b = [torch.empty_like(meas) for _ in range(2)]
        self.snap = [torch.empty_like(vol) for _ in range(2)]
        self.uploaded = [torch.cuda.Event() for _ in range(2)]
        self.consumed = [torch.cuda.Event() for _ in range(2)]
        self.snapped = [torch.cuda.Event() for _ in range(2)]
        self.read_back = [torch.cuda.Event() for _ in range(2)]
        self.k = 0


class SIRT_flatpanel:  # noqa: N801
    """An iterable SIRT reconstructor."""

    Config = _Config

    def __init__(self, config: _Config, volume: Volume, projs: fp.ProjectionSet) -> None:
        if projs.data is None:
            msg = "The provided ProjectionSet object has no data."
            raise ValueError(msg)
        if config.mode not in ("reference", "classical"):
            msg = f"unknown SIRT mode {config.mode!r}"
            raise ValueError(msg)
        self._config = config
        self._vol = volume
        self._meas = projs
        self._iterations = 0
        self._graph: torch.cuda.CUDAGraph | None = None
        self._graph_n = 0
        self._pipe: _HostPipeline | None = None
        self._config_fp_residual = fp.ConfigProject(multiply_before_adding=-1)
        sep = 0 if config.bp_soft_from_detedge_relrad is None else (1 - config.bp_soft_from_detedge_relrad)
        cyl = min(*volume.shape[:2]) / 2 * volume.voxwid
        p = projs.zeroed_copy(dtype=np.float32)  # the residual is FP32 whatever the measurement's type
        if config.mode == "reference":
            self._config_bp = fp.ConfigBackproject(
                fast_approx=config.fast_backproject,
                cyl_mask_rad=cyl,
                apply_summand_multiplier=True,
                soften_det_edges_proportion=sep,
            )
            self._precond = self._reference_preconditioner(volume, p, cyl, sep)
            self._rownorm = None
        else:
            self._config_bp = fp.ConfigBackproject(apply_summand_multiplier=True)
            self._precond, self._rownorm = self._classical_normalisers(volume, p)
        self._scratch = p

    # ------------------------------------------------------------------ setup
    def _reference_preconditioner(self, volume: Volume, p: fp.ProjectionSet, cyl: float, sep: float) -> Volume:
        """M = s' / (B A 1 + soft zero), masked (sirt_vram.py:83-118)."""
        M = volume.zeroed_copy()  # noqa: N806
        scale = 1 / float(np.mean(volume.shape))
        M.fill(1 * scale)
        M.soften_to_xy_cylinder(1)  # hard mask to the inscribed cylinder
        fp.project(fp.ConfigProject(), M, p, block=True)
        meanval = float(p.data.double().mean())
        p.data.div_(meanval / scale)
        scale /= meanval / scale
        M.fill(0)
        cfg = fp.ConfigBackproject(
            fast_approx=self._config.fast_backproject,
            cyl_mask_rad=cyl,
            apply_summand_multiplier=False,
            soften_det_edges_proportion=sep,
        )
        fp.backproject(cfg, M, p, block=True)
        M.invert(ignore_zeros=True, softmax_epsilon=0.1)
        M.multiply(scale)
        if self._config.soft_from_cylinder_relrad is not None:
            M.soften_to_xy_cylinder(self._config.soft_from_cylinder_relrad)
        return M

    def _classical_normalisers(self, volume: Volume, p: fp.ProjectionSet) -> tuple[Volume, torch.Tensor]:
        """C = 1/(B 1) on voxels, R = 1/(A 1) on rays (zero where the sums vanish)."""
        ones = volume.zeroed_copy()
        ones.fill(1.0)
        fp.project(fp.ConfigProject(), ones, p, block=True)
        rs = p.data
        R = torch.where(rs > 0, 1.0 / rs, torch.zeros_like(rs))  # noqa: N806
        C = volume.zeroed_copy()  # noqa: N806
        p.data.fill_(1.0)
        fp.backproject(fp.ConfigBackproject(), C, p, block=True)
        C.invert(ignore_zeros=True)
        p.data.zero_()
        return C, R

    # -------------------------------------------------------------- iteration
    def _step(self) -> None:
        """One iteration as two kernels: r = b - A x, then x += M (.) B r."""
        fp.project_residual(self._config_fp_residual, self._vol, self._scratch, self._meas.data)
        if self._rownorm is not None:
            self._scratch.data.mul_(self._rownorm)
        fp.backproject(self._config_bp, self._vol, self._scratch, summand_multiplier=self._precond)

    def iterate(self) -> None:
        """Perform one iteration (asynchronous on the current stream)."""
        self._step()
        self._iterations += 1

    def iterate_from_host(self, b_host: torch.Tensor, x_host: torch.Tensor | None = None) -> None:
        """One iteration whose measurement comes from host memory and whose
        result goes back to host memory, with both transfers overlapped with
        the neighbouring iterations' compute (asynchronous on the current stream).

        ``b_host``: this iteration's measurement b, a pinned host tensor of the
        projection data's shape. It is uploaded on an upload stream into one of
        two device buffers of this iterator (the ProjectionSet given to
        ``__init__`` is not touched); the iteration waits only for its own
        upload, so the next call's upload runs while this iteration computes.
        ``x_host``: a pinned host tensor of the volume's shape that receives the
        volume after this iteration: the volume is copied to one of two device
        snapshots (a device-to-device copy) and read back on a download stream
        while the next iteration runs. Keep ``b_host`` unchanged and read
        ``x_host`` only after :meth:`host_sync` (or a device synchronisation).
        """
        if tuple(b_host.shape) != tuple(self._meas.data.shape):
            msg = "b_host must have the projection data's shape"
            raise ValueError(msg)
        if x_host is not None and tuple(x_host.shape) != tuple(self._vol.data.shape):
            msg = "x_host must have the volume's shape"
            raise ValueError(msg)
        if self._pipe is None:
            self._pipe = _HostPipeline(self._meas.data, self._vol.data)
        pp = self._pipe
        i = pp.k % 2
        compute = torch.cuda.current_stream()
        with torch.cuda.stream(pp.up):
            pp.up.wait_event(pp.consumed[i])  # the iteration that read buffer i two calls ago is done with it
            pp.b[i].copy_(b_host, non_blocking=True)
            pp.b[i].record_stream(pp.up)
            pp.uploaded[i].record(pp.up)
        compute.wait_event(pp.uploaded[i])
        fp.project_residual(self._config_fp_residual, self._vol, self._scratch, pp.b[i])
        pp.consumed[i].record(compute)
        if self._rownorm is not None:
            self._scratch.data.mul_(self._rownorm)
        fp.backproject(self._config_bp, self._vol, self._scratch, summand_multiplier=self._precond)
        if x_host is not None:
            compute.wait_event(pp.read_back[i])  # snapshot i's previous read-back has ended
            pp.snap[i].copy_(self._vol.data)
            pp.snapped[i].record(compute)
            with torch.cuda.stream(pp.down):
                pp.down.wait_event(pp.snapped[i])
                x_host.copy_(pp.snap[i], non_blocking=True)
                pp.snap[i].record_stream(pp.down)
                pp.read_back[i].record(pp.down)
        pp.k += 1
        self._iterations += 1

    def host_sync(self) -> None:
        """Make the current stream wait for every transfer of :meth:`iterate_from_host` and block until done."""
        if self._pipe is not None:
            s = torch.cuda.current_stream()
            s.wait_stream(self._pipe.up)
            s.wait_stream(self._pipe.down)
        torch.cuda.current_stream().synchronize()

    def iterate_graph(self, n: int) -> None:
        """Perform ``n`` iterations by replaying one captured CUDA graph.

        The graph (2n kernel nodes, no host synchronisation) is captured on
        first use for a given ``n`` and replayed afterwards. Every kernel it
        launches has already run once in ``__init__``, so capture triggers no
        lazy module loading.
        """
        if n <= 0:
            return
        if self._graph is None or self._graph_n != n:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                for _ in range(n):
                    self._step()
            self._graph, self._graph_n = g, n
        self._graph.replay()
        self._iterations += n

    # ------------------------------------------------------------ accessors
    @property
    def volume(self) -> Volume:
        """The volume being reconstructed."""
        return self._vol

    @property
    def preconditioner(self) -> Volume:
        """The per-voxel multiplier M."""
        return self._precond

    @property
    def iterations(self) -> int:
        """Iterations performed so far."""
        return self._iterations

    def state_dict(self) -> dict:
        """Checkpoint: iterate, preconditioner, counter and config."""
        return {
            "x": self._vol.data.detach().cpu().clone(),
            "M": self._precond.data.detach().cpu().clone(),
            "R": None if self._rownorm is None else self._rownorm.detach().cpu().clone(),
            "iterations": self._iterations,
            "config": dataclasses.asdict(self._config),
        }

    def load_state_dict(self, sd: dict) -> None:
        """Resume from :meth:`state_dict`."""
        if sd["config"] != dataclasses.asdict(self._config):
            msg = "checkpoint was written with a different SIRT configuration"
            raise ValueError(msg)
        self._vol.data.copy_(sd["x"])
        self._precond.data.copy_(sd["M"])
        if sd["R"] is not None:
            self._rownorm = sd["R"].to(self._vol.data.device)
        self._iterations = int(sd["iterations"])
        self._graph = None
