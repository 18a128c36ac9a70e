"""Scan trajectories for synthetic workloads and tests.

* :func:`helical_scan` -- sources on a helix about the z axis with a flat
  detector facing them, the per-view layout of the reference's
  cone-cylinder geometry generator (src/aprict/scripts/make_geometry_cone_cyl.py:276-295:
  source (R cos t, R sin t, z), detector centre (-(L-R) cos t, -(L-R) sin t, z),
  u = pixwid (-sin t, cos t, 0), v = pixhei (0, 0, -1)), with z advancing by
  ``pitch`` detector heights (at the isocentre) per turn.
* :func:`jitter_views` -- per-view source/detector translation and a rigid
  detector rotation, for arbitrary (non-circular) geometry.
"""

from __future__ import annotations

import numpy as np

from .cb import flatpanel as fp


def helical_scan(
    *,
    n_views: int,
    R: float,  # noqa: N803
    L_minus_R: float,  # noqa: N803
    pix_at_iso: float,
    nu: int,
    nv: int,
    pitch: float,
    theta_start: float = 0.0,
    z_centre: float = 0.0,
) -> fp.ProjGeom:
    """A helical cone-beam scan covering one turn per ``n_views`` views."""
    mag = (R + L_minus_R) / R
    pix = pix_at_iso * mag
    t = theta_start + 2 * np.pi * np.arange(n_views) / n_views
    h_iso = nv * pix_at_iso
    z = z_centre + pitch * h_iso * (np.arange(n_views) / n_views - 0.5)
    src = np.stack([R * np.cos(t), R * np.sin(t), z], axis=1)
    det = np.stack([-L_minus_R * np.cos(t), -L_minus_R * np.sin(t), z], axis=1)
    u = pix * np.stack([-np.sin(t), np.cos(t), 0 * t], axis=1)
    v = np.broadcast_to(pix * np.array([0.0, 0.0, -1.0]), (n_views, 3)).copy()
    return fp.ProjGeom(source_pos=src, det_pos=det, det_uvec=u, det_vvec=v, nu=nu, nv=nv)


def cylinder_scan(
    *,
    n_views: int,
    R: float,  # noqa: N803
    L_minus_R: float,  # noqa: N803
    pix_at_iso: float,
    nu: int,
    nv: int,
    height: float,
    theta_start: float = 0.0,
    clockwise: bool = False,
) -> fp.ProjGeom:
    """Source points on a cylinder of radius R: heights evenly spaced over
    (-height/2, height/2) (ends excluded), angles stepping by the golden angle
    (sqrt(5) - 1) pi -- the GOLDEN_THETA trajectory of the reference's
    cone-cylinder geometry maker (scripts/make_geometry_cone_cyl.py:233-289)."""
    mag = (R + L_minus_R) / R
    pix = pix_at_iso * mag
    zs = np.linspace(-height / 2, height / 2, num=n_views + 2, endpoint=True)[1:-1]
    ts = theta_start + (-1 if clockwise else 1) * np.arange(n_views, dtype=np.float64) * (np.sqrt(5) - 1) * np.pi
    src = np.stack([R * np.cos(ts), R * np.sin(ts), zs], axis=1)
    det = np.stack([-L_minus_R * np.cos(ts), -L_minus_R * np.sin(ts), zs], axis=1)
    u = pix * np.stack([-np.sin(ts), np.cos(ts), 0 * ts], axis=1)
    v = np.broadcast_to(pix * np.array([0.0, 0.0, -1.0]), (n_views, 3)).copy()
    return fp.ProjGeom(source_pos=src, det_pos=det, det_uvec=u, det_vvec=v, nu=nu, nv=nv)


def jitter_views(rng: np.random.Generator, pg: fp.ProjGeom, mm: float = 2.0, deg: float = 0.5) -> fp.ProjGeom:
    """Per view: source and detector moved by up to +-mm along each axis, and
    the detector's u and v turned together (staying orthogonal) by up to +-deg
    about a random axis."""
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


def uneven_scans(
    rng: np.random.Generator,
    n_scans: int,
    *,
    edge: tuple[int, int] = (64, 320),
    views: tuple[int, int] = (90, 720),
    det: tuple[int, int] = (128, 768),
    voxwid: float = 0.5,
    R: float = 500.0,  # noqa: N803
    L_minus_R: float = 500.0,  # noqa: N803
) -> list[dict]:
    """Parameters of ``n_scans`` uneven scans: volume edge log-uniform in
    ``edge``, view count uniform in ``views``, square detector uniform in
    ``det``; circular or helical (pitch U(0.5, 1.5)) trajectories, all with
    per-view jitter of +-2 mm and +-0.5 degrees. The detector covers the
    volume's circumscribed cylinder at the isocentre."""
    out = []
    for _ in range(n_scans):
        n = int(round(np.exp(rng.uniform(np.log(edge[0]), np.log(edge[1])))))
        m = int(rng.integers(views[0], views[1] + 1))
        d = int(rng.integers(det[0], det[1] + 1))
        helical = bool(rng.random() < 0.5)
        pitch = float(rng.uniform(0.5, 1.5)) if helical else 0.0
        pix_at_iso = 1.5 * n * voxwid / d  # field of view 1.5x the volume edge
        out.append(dict(n=n, views=m, det=d, helical=helical, pitch=pitch, pix_at_iso=pix_at_iso, voxwid=voxwid,
                        R=R, L_minus_R=L_minus_R, theta0=float(rng.uniform(0, 2 * np.pi))))
    return out


def scan_geometry(rng: np.random.Generator, s: dict) -> fp.ProjGeom:
    """The jittered geometry of one :func:`uneven_scans` entry."""
    if s["helical"]:
        pg = helical_scan(n_views=s["views"], R=s["R"], L_minus_R=s["L_minus_R"], pix_at_iso=s["pix_at_iso"],
                          nu=s["det"], nv=s["det"], pitch=s["pitch"], theta_start=s["theta0"])
    else:
        pg = fp.ProjGeom.new_circular_scan(
            num_source_points=s["views"], R=s["R"], L_minus_R=s["L_minus_R"],
            pix_widhei_at_isocenter=(s["pix_at_iso"],) * 2, num_pix_widhei=(s["det"], s["det"]),
            theta_start=s["theta0"],
        )
    return jitter_views(rng, pg)


__all__ = ["helical_scan", "jitter_views", "scan_geometry", "uneven_scans"]
