"""Analytic projection of FORBILD phantoms (the ``FBVolume`` branch of ``project``).

The reference projects a FORBILD phantom with project_CB_FORBILD_shapes
(src/aprict/data/cusrc/CB_project_texture_chunked.cu:415-593) after pruning
the shapes to the bounding box of the scan on the host
(src/aprict/cb/flatpanel.py:1044-1045, 1088-1097). Here the shapes are
compiled once per phantom into canonical quadrics (FP64, on the host, by
``aprict_b200_forbild_compile``) and uploaded; every CTA culls them against
its own detector tile, so no host pruning is needed.

Modes: the reference's ConfigProject always resolves overlaps by "later
shapes win" (flatpanel.py:917-926); ``ConfigProject(overlap_addition=True)``
selects its additive mode, which sums rho times the *parametric* chord on the
source->pixel segment without the segment length (:556-560);
``additive_line_integral=True`` gives the additive line integral in length
units instead.
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _lib
from .. import _structs as S

SHAPE_TYPES = {
    "Box": 1, "Cone": 2, "Cone_x": 3, "Cone_y": 4, "Cone_z": 5, "Cylinder": 6, "Cylinder_x": 7, "Cylinder_y": 8,
    "Cylinder_z": 9, "Ellipsoid": 10, "Ellipsoid_free": 11, "Ellipt_Cyl": 12, "Sphere": 13, "Ellipt_Cyl_x": 14,
    "Ellipt_Cyl_y": 15, "Ellipt_Cyl_z": 16,
}  # src/aprict/cuda/structs/FORBILD_volumes.py:517-534


def compile_shapes(shapes: np.ndarray) -> np.ndarray:
    """FORBILD_Shape records -> aprict_quadric records (host, FP64)."""
    sh = np.ascontiguousarray(shapes.reshape(-1))
    if sh.dtype.itemsize != S.forbild_shape.itemsize:
        msg = "shapes must be 156-byte FORBILD_Shape records"
        raise ValueError(msg)
    out = np.zeros(len(sh), dtype=S.quadric)
    _lib.check(_lib.lib().aprict_b200_forbild_compile(sh.ctypes.data, len(sh), out.ctypes.data), "forbild_compile")
    return out


def shape_bboxes(shapes: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(mins, maxs), each (N, 3): world bounding boxes of the (unclipped) shapes."""
    q = compile_shapes(shapes)
    return q["c"] - q["bb_half"], q["c"] + q["bb_half"]


class _Compiled:
    """Device copy of a phantom's compiled shapes, cached on the FBVolume."""

    def __init__(self, shapes: np.ndarray) -> None:
        self.host = compile_shapes(shapes)
        raw = self.host.view(np.uint8).reshape(-1)
        self.dev = torch.from_numpy(raw.copy()).cuda() if raw.size else None
        self.n = len(self.host)


def _compiled(volume: object) -> _Compiled:
    cache = getattr(volume, "_compiled", None)
    if cache is None or cache[0] is not volume.shapes:
        volume._compiled = (volume.shapes, _Compiled(volume.shapes))
    return volume._compiled[1]


def project_shapes(config: object, volume: object, projs: object) -> None:
    """Accumulate the analytic projection of ``volume`` (an FBVolume) into ``projs``."""
    from .flatpanel import _leading_slices, _stream, _view_args  # noqa: PLC0415

    comp = _compiled(volume)
    if comp.n == 0 or comp.dev is None:
        return
    cfg = config.contents
    if config.overlap_addition:
        mode = 2 if getattr(config, "additive_line_integral", False) else 1
    else:
        mode = 0
    counter = projs.out_of_mem_counter
    for it, first in _leading_slices(projs):
        specs, pd, dptr = _view_args(projs, it, first)
        _lib.check(
            _lib.lib().aprict_b200_project_forbild(
                specs, _lib.ptr(pd), dptr, comp.dev.data_ptr(), comp.n, float(cfg["multiply_before_adding"]),
                int(cfg["ssu"]), int(cfg["ssv"]), mode, counter.data_ptr(), None, _stream(),
            ),
            "project (FORBILD)",
        )
