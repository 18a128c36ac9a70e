"""Seeded synthetic phantoms for tests and benchmarks.

The reference builds phantoms from FORBILD ``.pha`` files
(src/aprict/phantoms/FORBILD_phantoms.py) and voxelises them with "last shape
wins" semantics (src/aprict/data/cusrc/sample_FORBILD_volumes.cu:96-100).
The workloads here use random ellipsoids whose densities ADD, voxelised at
voxel centres; random orientations are orthonormalised as in the reference's
Ellipsoid_free tests (src/aprict/tests/cuda_kernels/test_project_cb_FORBILD_shapes.py:594-612).
"""

from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass(frozen=True)
class Ellipsoid:
    """An ellipsoid with centre ``c``, semi-axes ``a`` along the rows of ``rot``, density ``rho``."""

    c: np.ndarray
    a: np.ndarray
    rot: np.ndarray  # (3,3) orthonormal rows: the local x, y, z axes
    rho: float


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """A random orthonormal frame (rows) from Gram-Schmidt of Gaussian vectors."""
    m = rng.standard_normal((3, 3))
    q, r = np.linalg.qr(m.T)
    q = q * np.sign(np.diag(r))[None, :]
    return q.T


def random_ellipsoids(
    rng: np.random.Generator,
    n: int,
    *,
    shape: tuple[int, int, int],
    voxwid: float,
    pos_c: np.ndarray | tuple[float, float, float] = (0.0, 0.0, 0.0),
    semi_axes_vox: tuple[float, float] = (5.0, 40.0),
    rho: tuple[float, float] = (0.01, 0.1),
    inner: float = 0.8,
) -> list[Ellipsoid]:
    """``n`` ellipsoids with centres uniform in the inner ``inner`` fraction of the box."""
    pos_c = np.asarray(pos_c, dtype=np.float64)
    half = 0.5 * np.asarray(shape, dtype=np.float64) * voxwid
    out = []
    for _ in range(n):
        c = pos_c + rng.uniform(-inner, inner, size=3) * half
        a = rng.uniform(semi_axes_vox[0], semi_axes_vox[1], size=3) * voxwid
        out.append(Ellipsoid(c=c, a=a, rot=random_rotation(rng), rho=float(rng.uniform(rho[0], rho[1]))))
    return out


def voxelize(
    ellipsoids: list[Ellipsoid],
    shape: tuple[int, int, int],
    voxwid: float,
    pos_c: np.ndarray | tuple[float, float, float] = (0.0, 0.0, 0.0),
) -> np.ndarray:
    """Additive point-sampling at voxel centres -> float32 (X,Y,Z), C order."""
    pos_c = np.asarray(pos_c, dtype=np.float64)
    axes = [pos_c[i] + voxwid * (np.arange(shape[i], dtype=np.float64) - (shape[i] - 1) / 2) for i in range(3)]
    vol = np.zeros(shape, dtype=np.float32)
    for e in ellipsoids:
        # Bounding box of the ellipsoid, in index space, to keep this cheap.
        ext = np.sqrt(((e.rot * e.a[:, None]) ** 2).sum(axis=0))
        sl = []
        for i in range(3):
            lo = np.searchsorted(axes[i], e.c[i] - ext[i], side="left")
            hi = np.searchsorted(axes[i], e.c[i] + ext[i], side="right")
            sl.append(slice(lo, hi))
        if any(s.start >= s.stop for s in sl):
            continue
        X, Y, Z = np.meshgrid(axes[0][sl[0]], axes[1][sl[1]], axes[2][sl[2]], indexing="ij")
        d = np.stack([X - e.c[0], Y - e.c[1], Z - e.c[2]], axis=-1)
        loc = d @ e.rot.T / e.a
        inside = (loc**2).sum(axis=-1) <= 1.0
        vol[sl[0], sl[1], sl[2]] += np.float32(e.rho) * inside
    return vol


def ellipsoid_volume(
    seed: int,
    n: int,
    shape: tuple[int, int, int],
    voxwid: float,
    *,
    semi_axes_vox: tuple[float, float] = (5.0, 40.0),
    rho: tuple[float, float] = (0.01, 0.1),
) -> np.ndarray:
    """A seeded additive random-ellipsoid volume (the workloads' phantom)."""
    rng = np.random.default_rng(seed)
    return voxelize(random_ellipsoids(rng, n, shape=shape, voxwid=voxwid, semi_axes_vox=semi_axes_vox, rho=rho), shape, voxwid)


def _unit(v: np.ndarray) -> np.ndarray:
    return v / np.linalg.norm(v)


def random_quadric_phantom(
    seed: int,
    *,
    n_ellipsoids: int = 60,
    n_cylinders: int = 40,
    radius: float = 100.0,
    rho: tuple[float, float] = (-0.2, 1.0),
    size: tuple[float, float] = (5.0, 40.0),
    max_clips: int = 3,
) -> np.ndarray:
    """FORBILD_Shape records: free ellipsoids (type 11) then elliptic cylinders (type 12).

    Each shape has 0..max_clips random clip planes through a point near its
    centre, a density uniform in ``rho``, and lies inside a sphere of
    ``radius`` (the quadric-phantom workload: 60 + 40 shapes in 200 mm).
    """
    from ._structs import forbild_shape  # noqa: PLC0415

    rng = np.random.default_rng(seed)
    n = n_ellipsoids + n_cylinders
    out = np.zeros(n, dtype=forbild_shape)
    for i in range(n):
        frame = random_rotation(rng)
        semi = rng.uniform(size[0], size[1], size=3)
        ext = float(np.max(semi))
        if i >= n_ellipsoids:
            ext = float(np.hypot(max(semi[0], semi[1]), semi[2]))
        dist = rng.uniform(0, max(radius - ext, 0.0))
        c = _unit(rng.standard_normal(3)) * dist
        rec = out[i]
        rec["rho"] = rng.uniform(*rho)
        rec["x"], rec["y"], rec["z"] = c
        if i < n_ellipsoids:
            rec["type"] = 11
            rec["dx"], rec["dy"], rec["dz"] = semi
            rec["a_x"] = tuple(frame[0])
            rec["a_y"] = tuple(frame[1])
            rec["a_z"] = tuple(frame[2])
        else:
            rec["type"] = 12
            rec["dx"], rec["dy"] = semi[0], semi[1]
            rec["l"] = 2 * semi[2]
            rec["a_x"] = tuple(frame[0])
            rec["a_y"] = tuple(frame[1])
            rec["axis"] = tuple(frame[2])
        for k in range(int(rng.integers(0, max_clips + 1))):
            a = _unit(rng.standard_normal(3))
            d = float(a @ c + rng.uniform(-0.5, 0.5) * ext)
            cas = rec[f"cas{k + 1}"]
            cas["axis"] = tuple(a)
            cas["dotprod"] = d
            cas["mode"] = int(rng.integers(1, 3))
    return out
