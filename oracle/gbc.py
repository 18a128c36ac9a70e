"""FP64 restatement of the reference's GBC reconstruction pieces. TEST
INFRASTRUCTURE: only tests/ import this module, as the checker; nothing in
the product path uses it.

* ``soft_window`` / ``gbc_weight``: cossq_soft and _GBC_weightfun
  (src/aprict/data/cusrc/CB_backproject.cu:273-311, 736-787);
* ``backproject_gbc``: _backproject_CB_getval_GBC_cyl and
  backproject_CB_voltex_GBC_cyl (:788-905, 1030-1105) with the detector
  coordinate of get_projected_detector_coords (geometry.h:24-56) and the
  nearest / bilinear rules of get_zero_interp / get_bilinear_interp
  (CB_backproject.cu:221-271);
* ``weight_integral``: get_GBC_weight_integ (:1108-1168);
* ``conebeam_kfactor`` / ``ramp_filter_conebeam``: _conebeam_kfactor_unchunked
  and ramp_filter_conebeam (src/aprict/gbc/filters.py:59-147, 256-504), with
  NumPy's FFT;
* ``add_upsampled``: the low-resolution correction of ramp_filter_conebeam
  (filters.py:403-455), the order-1 "nearest" interpolation restated (tests
  pin it against scipy.ndimage.map_coordinates, the published definition
  behind the reference's cupyx call).
"""

from __future__ import annotations

import numpy as np


def soft_window(a: float, b: float, c: np.ndarray) -> np.ndarray:
    """s(a, b; c): 0 for |c| > a, 1 for |c| < a - b, else 3x^2 - 2x^3 with x = gamma sin|c| - chi."""
    c = np.abs(np.asarray(c, dtype=np.float64))
    gamma = 1.0 / (np.sin(a - b) - np.sin(a))
    chi = gamma * np.sin(a)
    x = gamma * np.sin(c) - chi
    mid = np.clip(3 * x * x - 2 * x * x * x, 0.0, 1.0)
    return np.where(c > a, 0.0, np.where(c < a - b, 1.0, mid))


def gbc_weight(R: float, vox: np.ndarray, src: np.ndarray, soft: tuple[float, float, float, float]) -> np.ndarray:  # noqa: N803
    """GBC weight for voxel positions vox (..., 3) and sources src (..., 3); soft = (v, v_span, h, h_span)."""
    vox = np.asarray(vox, np.float64)
    src = np.asarray(src, np.float64)
    r = vox - src
    lnorm = np.hypot(src[..., 0], src[..., 1])
    Z = (r[..., 0] * -src[..., 0] + r[..., 1] * -src[..., 1]) / lnorm  # noqa: N806
    ell = np.hypot(r[..., 0], r[..., 1]) / R
    with np.errstate(divide="ignore", invalid="ignore"):
        c = np.clip(np.abs((Z / R) / ell), 0.0, 1.0)
    c = np.where(np.isnan(c), 1.0, c)
    d = c - ell
    th = np.arctan2(r[..., 2] / R, ell)
    w = np.cos(th) ** 3 * c / np.maximum(1e-9, c * c + d * d)
    return w * soft_window(soft[0], soft[1], th) * soft_window(soft[2], soft[3], np.arccos(c))


def detector_coords(spec: np.void, pts: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Fractional pixel indices (from the corner pixel's centre) of points pts (..., 3) (geometry.h:24-56)."""
    s = np.array(spec["source_pos"].tolist(), np.float64)
    P = np.array(spec["det_pos"].tolist(), np.float64)  # noqa: N806
    U = np.array(spec["det_u"].tolist(), np.float64)  # noqa: N806
    V = np.array(spec["det_v"].tolist(), np.float64)  # noqa: N806
    n = np.cross(U, V)
    lam = np.dot(P - s, n) / ((pts - s) @ n)
    p = s + (pts - s) * lam[..., None] - P
    fu = (p @ U) / np.dot(U, U) + (int(spec["nu"]) - 1) / 2
    fv = (p @ V) / np.dot(V, V) + (int(spec["nv"]) - 1) / 2
    return fu, fv


def _sample(img: np.ndarray, fu: np.ndarray, fv: np.ndarray, linear: bool) -> np.ndarray:
    nu, nv = img.shape

    def get(i, j):
        ok = (i >= 0) & (i < nu) & (j >= 0) & (j < nv)
        return np.where(ok, img[np.clip(i, 0, nu - 1), np.clip(j, 0, nv - 1)], 0.0)

    if not linear:
        return get(np.floor(fu + 0.5).astype(np.int64), np.floor(fv + 0.5).astype(np.int64))
    out_range = (fu <= -1) | (fv <= -1) | (fu >= nu) | (fv >= nv)
    i0, j0 = np.floor(fu).astype(np.int64), np.floor(fv).astype(np.int64)
    fx, fy = fu - i0, fv - j0
    t1 = get(i0, j0) * (1 - fx) + get(i0 + 1, j0) * fx
    t2 = get(i0, j0 + 1) * (1 - fx) + get(i0 + 1, j0 + 1) * fx
    return np.where(out_range, 0.0, t1 * (1 - fy) + t2 * fy)


def backproject_gbc(specs: np.ndarray, projs: np.ndarray, shape: tuple[int, int, int], voxwid: float,
                    corner: np.ndarray, *, R: float, soft: tuple[float, float, float, float],  # noqa: N803
                    linear: bool = False, ss: tuple[int, int, int] = (1, 1, 1),
                    mult: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
    """(volume, weight sums) added by the GBC backprojection of projs (M, nu, nv), C order (x, y, z)."""
    nx, ny, nz = shape
    idx = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).astype(np.float64)
    corner = np.asarray(corner, np.float64)
    acc = np.zeros(shape)
    acc2 = np.zeros(shape)
    subs = [(i, j, k) for i in range(ss[0]) for j in range(ss[1]) for k in range(ss[2])]
    for si in subs:
        off = np.array([-0.5 + (0.5 + si[a]) / ss[a] for a in range(3)])
        pts = corner + (idx + 0.5 + off) * voxwid
        for m, sp in enumerate(specs):
            src = np.broadcast_to(np.array(sp["source_pos"].tolist(), np.float64), pts.shape)
            w = gbc_weight(R, pts, src, soft)
            acc2 += w
            fu, fv = detector_coords(sp, pts)
            acc += np.where(w != 0, _sample(np.asarray(projs[m], np.float64), fu, fv, linear) * w, 0.0)
    n_sub = len(subs)
    acc /= n_sub
    acc2 /= n_sub
    if mult is not None:
        acc = acc * mult
        acc2 = acc2 * mult
    return acc, acc2


def weight_integral(r_on_R: np.ndarray, soft: tuple[float, float, float, float], num_z: int, num_ang: int) -> np.ndarray:  # noqa: N803
    """Expected weight sums at radii r_on_R over a cylindrical locus (get_GBC_weight_integ)."""
    r_on_R = np.asarray(r_on_R, np.float64)  # noqa: N806
    maxz = np.tan(soft[0]) * (1 + r_on_R[-1])
    z = maxz * np.arange(num_z) / (num_z - 1)
    t = np.arange(num_ang) / num_ang * np.pi
    zz, tt = np.meshgrid(z, t, indexing="ij")
    src = np.stack([np.cos(tt), np.sin(tt), zz], -1)
    half = np.where(np.arange(num_z) == 0, 0.5, 1.0)[:, None]
    mult = 4 * maxz * np.pi / (num_z * num_ang)
    out = np.empty(len(r_on_R))
    for i, r in enumerate(r_on_R):
        vox = np.broadcast_to(np.array([r, 0.0, 0.0]), src.shape)
        out[i] = np.sum(gbc_weight(1.0, vox, src, soft) * half) * mult
    return out


def conebeam_kfactor(theta: np.ndarray, cone: float, soft: float) -> np.ndarray:
    """k-factor of the softened Colsher window (filters.py:59-147)."""
    th = np.abs(np.asarray(theta, np.float64))
    if cone == np.pi:
        return np.full_like(th, 2 * np.pi)
    h = cone / 2 - soft
    mask = (h < th) & (th < np.pi - h)
    out = np.full_like(th, 2 * np.pi)
    s = np.sin(th[mask])
    gamma = 1 / (np.sin(cone / 2 - soft) - np.sin(cone / 2))
    chi = gamma * np.sin(cone / 2)
    alpha = 0.0 if h <= 0 else np.clip(np.sin(h) / s, 0, 1)
    beta = np.clip(np.where(np.sin(cone / 2) >= s, 1.0, np.sin(cone / 2) / s), 0, 1)
    t1 = np.arcsin(beta) - np.arcsin(alpha)
    t2 = np.sqrt(1 - beta**2)
    t3 = np.sqrt(1 - alpha**2)
    v = t1 * 4 * chi**2 * (3 + 2 * chi) + 4 * np.arcsin(alpha)
    v = v + s * (24 * gamma * chi * (1 + chi) * (t2 - t3))
    v = v + s**2 * (6 * gamma**2 * (1 + 2 * chi) * (t1 - beta * t2 + alpha * t3))
    v = v + s**3 * (-2 / 3 * gamma**3 * (-9 * (t2 - t3) + (np.cos(3 * np.arcsin(beta)) - np.cos(3 * np.arcsin(alpha)))))
    out[mask] = v
    return out


def add_upsampled(out: np.ndarray, low: np.ndarray, d: int) -> np.ndarray:
    """out += order-1 interpolation of low at idx / d - 1/2 + 1/(2d), neighbours clamped (mode "nearest")."""
    coords = [np.arange(n) / d - 0.5 + 1 / d / 2 for n in out.shape]
    res = np.zeros(out.shape)
    parts = []
    for a, c in enumerate(coords):
        f = np.floor(c)
        t = c - f
        i0 = np.clip(f.astype(np.int64), 0, low.shape[a] - 1)
        i1 = np.clip(f.astype(np.int64) + 1, 0, low.shape[a] - 1)
        parts.append((i0, i1, t))
    (x0, x1, tx), (y0, y1, ty), (z0, z1, tz) = parts
    for ax, wx in ((x0, 1 - tx), (x1, tx)):
        for ay, wy in ((y0, 1 - ty), (y1, ty)):
            for az, wz in ((z0, 1 - tz), (z1, tz)):
                res += wx[:, None, None] * wy[None, :, None] * wz[None, None, :] * low[np.ix_(ax, ay, az)]
    return out + res


def ramp_filter_conebeam(arr: np.ndarray, voxel_len: float, cone: float, soft: float,
                         lowres: np.ndarray | None = None, extra_multiplier: float = 1.0) -> np.ndarray:
    """The cone-beam ramp filter of a (n0, n1, n2) volume (filters.py:256-504), FP64."""
    a = np.asarray(arr, np.float64)
    n0, n1, n2 = a.shape
    f = np.fft.rfftn(a, norm="ortho")
    f0 = np.fft.fftfreq(n0)[:, None, None]
    f1 = np.fft.fftfreq(n1)[None, :, None]
    f2 = np.fft.rfftfreq(n2)[None, None, :]
    lat2 = f0**2 + f1**2
    mult = extra_multiplier / voxel_len
    if cone == 0:
        f = f * (np.sqrt(lat2) * mult)
    else:
        f = f * (np.sqrt(lat2 + f2**2) * mult)
        th = np.abs(np.pi / 2 - np.arctan2(np.broadcast_to(f2, f.shape), np.sqrt(np.broadcast_to(lat2, f.shape))))
        f = f / conebeam_kfactor(th, cone, soft)
    f = f * np.sinc(f0) * np.sinc(f1) * np.sinc(f2)
    f[0, 0, 0] = 0
    out = np.fft.irfftn(f, s=(n0, n1, n2), axes=(0, 1, 2), norm="ortho")
    if lowres is not None:
        out = add_upsampled(out, np.asarray(lowres, np.float64), n0 // lowres.shape[0])
    return out


def gbc_cone_cyl(specs: np.ndarray, projs: np.ndarray, volshape: tuple[int, int, int], voxwid: float,
                 volpos: tuple[float, float, float], *, R: float, L: float, pixwid: float, nu: int, nv: int,  # noqa: N803
                 zs: np.ndarray, n: int, f1: float, f2: float, eps: float, softspan_v: float, softspan_h: float,
                 linear: bool, num_z: int, num_ang: int) -> np.ndarray:
    """The GBC reconstruction driver (recon_cbfp_cyl_gbc.py:649-1380) on one volume
    (no z slabs), every view within reach of the volume."""
    import math  # noqa: PLC0415

    padded = tuple(n * (4 + math.ceil(s * f1 / n)) for s in volshape)
    padded = tuple(p if (p - s) % 2 == 0 else p + n for s, p in zip(volshape, padded))
    pads = tuple((p - s) // 2 for s, p in zip(volshape, padded))
    mini = tuple(math.ceil(s * f2 / n) for s in volshape)
    mini = tuple(max(m, p // n) for p, m in zip(padded, mini))
    mini = tuple(m if (m - p // n) % 2 == 0 else m + 1 for p, m in zip(padded, mini))
    mpads = tuple((m - p // n) // 2 for p, m in zip(padded, mini))
    vtv = np.arctan2(nv * pixwid / 2 - pixwid / 2, np.sqrt(L**2 + (nu * pixwid / 2 - pixwid / 2) ** 2))
    vth = np.arctan2(nu * pixwid / 2 - pixwid / 2, L)
    soft = (vtv, softspan_v, vth, softspan_h)
    mu = len(specs) / (2 * np.pi * R * (zs.max() - zs.min()))

    def corner_and_centres(shape, vw):
        c = np.asarray(volpos, np.float64) - vw * np.array(shape) / 2
        xs = [volpos[a] + vw * (np.arange(shape[a]) - (shape[a] - 1) / 2) for a in range(3)]
        return c, xs

    def recon(shape, vw):
        corner, xs = corner_and_centres(shape, vw)
        v, ws = backproject_gbc(specs, projs, shape, vw, corner, R=R, soft=soft, linear=linear)
        v, ws = v / (mu * R**2), ws / (mu * R**2)
        rel = np.sqrt(xs[0][:, None] ** 2 + xs[1][None, :] ** 2) / R
        r_in = np.linspace(rel.min(), rel.max(), num=2 * max(shape[0], shape[1]))
        integ = np.interp(rel, r_in, weight_integral(r_in, soft, num_z, num_ang))
        ws = ws * (1 / integ)[:, :, None]
        if eps > 0:
            ws = ws + eps * np.exp(-ws / eps)
        return v * (1 / ws)

    full = recon(padded, voxwid)
    small = recon(mini, voxwid * n)
    cone = 2 * vtv
    crop_m = tuple(slice(p, (-p) or None) for p in mpads)
    corr = ramp_filter_conebeam(small, voxwid * n, cone, softspan_v)[crop_m] - ramp_filter_conebeam(
        small[crop_m], voxwid * n, cone, softspan_v)
    out = ramp_filter_conebeam(full, voxwid, cone, softspan_v, lowres=corr)
    c = out[2 * n : -2 * n, 2 * n : -2 * n, 2 * n : -2 * n]
    dc = 0.25 * (c[:, 0, :].mean() + c[:, -1, :].mean() + c[0, :, :].mean() + c[-1, :, :].mean())
    out = out - dc
    return out[tuple(slice(p, (-p) or None) for p in pads)]
