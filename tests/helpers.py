"""Shared helpers for the parity tests (geometries, comparisons)."""

from __future__ import annotations

import numpy as np

from aprict_b200.cb import flatpanel as fp


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def circular(n_views: int, R: float, LmR: float, pix: float, nu: int, nv: int, theta0: float = 0.0123) -> fp.ProjGeom:
    """A circular scan; theta0 and a non-round pixel pitch keep voxel centres off exact half-pixel ties."""
    return fp.ProjGeom.new_circular_scan(
        num_source_points=n_views,
        R=R,
        L_minus_R=LmR,
        pix_widhei_at_isocenter=(pix, pix),
        num_pix_widhei=(nu, nv),
        theta_start=theta0,
    )


def jittered(rng: np.random.Generator, pg: fp.ProjGeom, mm: float = 2.0, deg: float = 0.5) -> fp.ProjGeom:
    """Per-view source/detector jitter: +-mm translations, +-deg rotation of the detector vectors."""
    m = pg.num_projs

    def rot(v: np.ndarray) -> np.ndarray:
        out = np.empty((m, 3), dtype=np.float64)
        for i in range(m):
            ax = rng.standard_normal(3)
            ax /= np.linalg.norm(ax)
            ang = np.deg2rad(rng.uniform(-deg, deg))
            K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
            Rm = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K
            out[i] = Rm @ np.broadcast_to(v, (m, 3))[i]
        return out

    return fp.ProjGeom(
        source_pos=pg.source_pos + rng.uniform(-mm, mm, size=(m, 3)),
        det_pos=pg.det_pos + rng.uniform(-mm, mm, size=(m, 3)),
        det_uvec=rot(pg.det_uvec),
        det_vvec=rot(pg.det_vvec),
        nu=pg.nu,
        nv=pg.nv,
    )
