"""Differentiable Siddon projection for PyTorch.

``SiddonProjectFn`` is a ``torch.autograd.Function`` whose forward is the
Siddon projector (``aprict_b200_project_siddon``) and whose backward is its
matched adjoint, the ray-driven scatter with the same intersection lengths
(``aprict_b200_backproject_scatter``). The operator is linear, so nothing is
saved for backward: grad_x = A^T grad_out. This makes
``0.5 * ||A x - b||^2`` differentiable with the gradient A^T (A x - b) -- the
quantity the reference's Landweber iteration with ``--exact-adjoint``
steps along (src/aprict/iterators/landweber_vram.py:221-260).
"""

from __future__ import annotations

import numpy as np
import torch

from .cb import flatpanel as fp
from .volume import Volume


class SiddonProjector:
    """A fixed geometry (scan + voxel grid) to project tensors with, differentiably."""

    def __init__(
        self,
        pg: fp.ProjGeom,
        shape: tuple[int, int, int],
        *,
        voxwid: float,
        pos_c: tuple[float, float, float] | np.ndarray = (0.0, 0.0, 0.0),
        config: fp.ConfigProject | None = None,
    ) -> None:
        self.pg = pg
        self.shape = tuple(int(s) for s in shape)
        self.voxwid = float(voxwid)
        self.pos_c = np.asarray(pos_c, dtype=np.float32)
        self.config = config or fp.ConfigProject()
        self._ps = fp.ProjectionSet(pg, data=None)
        self.data_shape = tuple(self._ps.proj_specs.shape) + (int(pg.nu.flat[0]), int(pg.nv.flat[0]))

    def _volume(self, x: torch.Tensor) -> Volume:
        if tuple(x.shape) != self.shape:
            msg = f"expected a volume of shape {self.shape}, got {tuple(x.shape)}"
            raise ValueError(msg)
        return Volume.from_tensor(x.contiguous(), voxwid=self.voxwid, pos_c=self.pos_c)

    def forward_raw(self, x: torch.Tensor) -> torch.Tensor:
        """A x (no autograd)."""
        out = torch.zeros(self.data_shape, dtype=torch.float32, device=x.device)
        ps = fp.ProjectionSet(self.pg, data=out)
        ps._specs_dev = self._ps.specs_device()  # noqa: SLF001
        fp.project(self.config, self._volume(x), ps)
        return out

    def adjoint_raw(self, y: torch.Tensor) -> torch.Tensor:
        """A^T y (no autograd), the exact transpose of :meth:`forward_raw`."""
        out = torch.zeros(self.shape, dtype=torch.float32, device=y.device)
        ps = fp.ProjectionSet(self.pg, data=y.contiguous())
        ps._specs_dev = self._ps.specs_device()  # noqa: SLF001
        fp.backproject_adjoint(self.config, Volume.from_tensor(out, voxwid=self.voxwid, pos_c=self.pos_c), ps)
        return out

    def __call__(self, x: torch.Tensor) -> torch.Tensor:
        return SiddonProjectFn.apply(x, self)


class SiddonProjectFn(torch.autograd.Function):
    """y = A x with backward grad_x = A^T grad_y (matched adjoint)."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, proj: SiddonProjector) -> torch.Tensor:  # noqa: ANN001
        if x.dtype != torch.float32 or not x.is_cuda:
            msg = "SiddonProjectFn needs a float32 CUDA tensor"
            raise ValueError(msg)
        ctx.proj = proj
        return proj.forward_raw(x.detach())

    @staticmethod
    def backward(ctx, grad_y: torch.Tensor) -> tuple[torch.Tensor, None]:  # noqa: ANN001
        return SiddonAdjointFn.apply(grad_y, ctx.proj), None


class SiddonAdjointFn(torch.autograd.Function):
    """x = A^T y with backward grad_y = A grad_x (so double backward works too)."""

    @staticmethod
    def forward(ctx, y: torch.Tensor, proj: SiddonProjector) -> torch.Tensor:  # noqa: ANN001
        ctx.proj = proj
        return proj.adjoint_raw(y.detach().float())

    @staticmethod
    def backward(ctx, grad_x: torch.Tensor) -> tuple[torch.Tensor, None]:  # noqa: ANN001
        return SiddonProjectFn.apply(grad_x.contiguous(), ctx.proj), None


def project_differentiable(
    x: torch.Tensor,
    pg: fp.ProjGeom,
    *,
    voxwid: float,
    pos_c: tuple[float, float, float] | np.ndarray = (0.0, 0.0, 0.0),
    config: fp.ConfigProject | None = None,
) -> torch.Tensor:
    """A x for a (X,Y,Z) float32 CUDA tensor, differentiable with the matched adjoint."""
    return SiddonProjector(pg, tuple(x.shape), voxwid=voxwid, pos_c=pos_c, config=config)(x)


__all__ = ["SiddonAdjointFn", "SiddonProjectFn", "SiddonProjector", "project_differentiable"]
