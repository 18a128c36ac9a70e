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
    """Per-view jitter: +-mm translations of source and detector, and a rigid
    rotation of the detector (u and v turned together, so they stay orthogonal)
    by up to +-deg about a random axis."""
    m = pg.num_projs
    U = np.broadcast_to(pg.det_uvec, (m, 3)).astype(np.float64)  # noqa: N806
    V = np.broadcast_to(pg.det_vvec, (m, 3)).astype(np.float64)  # noqa: N806
    Ur, Vr = np.empty_like(U), np.empty_like(V)  # noqa: N806
    for i in range(m):
        ax = rng.standard_normal(3)
        ax /= np.linalg.norm(ax)
        ang = np.deg2rad(rng.uniform(-deg, deg))
        K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])  # noqa: N806
        Rm = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K  # noqa: N806
        Ur[i], Vr[i] = Rm @ U[i], Rm @ V[i]
    return fp.ProjGeom(
        source_pos=pg.source_pos + rng.uniform(-mm, mm, size=(m, 3)),
        det_pos=pg.det_pos + rng.uniform(-mm, mm, size=(m, 3)),
        det_uvec=Ur,
        det_vvec=Vr,
        nu=pg.nu,
        nv=pg.nv,
    )


def random_shapes_all_types(rng: np.random.Generator, n: int, *, radius: float = 40.0, types: tuple[int, ...] | None = None) -> np.ndarray:
    """Random FORBILD_Shape records of every type (1..16), with 0-3 clip planes each."""
    from aprict_b200 import _structs as S
    from aprict_b200.phantoms import random_rotation

    types = types or tuple(range(1, 17))
    out = np.zeros(n, dtype=S.forbild_shape)
    for i in range(n):
        t = types[i % len(types)]
        rec = out[i]
        rec["type"] = t
        rec["rho"] = rng.uniform(-0.2, 1.0)
        c = rng.uniform(-radius, radius, size=3) * 0.6
        rec["x"], rec["y"], rec["z"] = c
        a, b, cc = rng.uniform(3, 15, size=3)
        rec["dx"], rec["dy"], rec["dz"] = a, b, cc
        rec["r"] = a
        rec["r1"], rec["r2"] = rng.uniform(0, 12), rng.uniform(2, 12)
        rec["l"] = rng.uniform(5, 30)
        f = random_rotation(rng)
        rec["a_x"], rec["a_y"], rec["a_z"] = tuple(f[0]), tuple(f[1]), tuple(f[2])
        rec["axis"] = tuple(f[2])
        for k in range(int(rng.integers(0, 4))):
            ax = rng.standard_normal(3)
            ax /= np.linalg.norm(ax)
            cas = rec[f"cas{k + 1}"]
            cas["axis"] = tuple(ax)
            cas["dotprod"] = float(ax @ c + rng.uniform(-5, 5))
            cas["mode"] = int(rng.integers(1, 3))
    return out
