"""The FP64 oracle's count of nearest-pixel choices it cannot settle (CPU only).

A circular scan with an even detector width puts the detector's centre-column
boundary on the plane through the source and the rotation axis; at a view
angle of 45 degrees that plane holds the voxel centres of one diagonal of a
cubic volume, whose nearest-pixel choice is then a tie in real arithmetic. The
counter must find exactly those voxels at that view, none at a view angle off
the symmetric ones, and one tie per diagonal voxel.
"""

from __future__ import annotations

import numpy as np

from aprict_b200.cb import flatpanel as fp
from oracle import oracle as O


def _views(theta: float) -> np.ndarray:
    pg = fp.ProjGeom.new_circular_scan(num_source_points=1, R=200.0, L_minus_R=200.0,
                                       pix_widhei_at_isocenter=(0.8, 0.8), num_pix_widhei=(48, 48),
                                       theta_start=theta)
    return pg.to_proj_spec_array()


def test_ties_on_the_diagonal_plane_at_45_degrees() -> None:
    n = 24
    cfg = fp.ConfigBackproject(fast_approx=True)
    corner = -np.array((n, n, n), np.float32) / 2
    c = O.bp_nearest_ties(_views(np.pi / 4), (n, n, n), cfg.contents, voxwid=1.0, corner=corner)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    # source direction (1, 1)/sqrt2: the plane through it and the z axis holds x == y
    diag = (i == j)[:, :, None] & np.ones(n, bool)[None, None, :]
    assert np.array_equal(c > 0, diag)
    assert c[diag].max() == 1


def test_no_ties_off_the_symmetric_angles() -> None:
    n = 24
    cfg = fp.ConfigBackproject(fast_approx=True)
    corner = -np.array((n, n, n), np.float32) / 2
    c = O.bp_nearest_ties(_views(0.3), (n, n, n), cfg.contents, voxwid=1.0, corner=corner)
    assert c.sum() == 0
