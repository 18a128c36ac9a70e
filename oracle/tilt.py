"""FP64 restatement of the reference's cone-cylinder ("tilted") projection
filter and FBP driver. TEST INFRASTRUCTURE: only tests/ import this module,
as the checker; nothing in the product path uses it.

Follows FBPFilterer (src/aprict/cb/ramp_filter.py:333-886):

* rotation sampling: one ``rng.random()`` per projection,
  ``angle = lo + (hi - lo) * u`` stored as float32 (``uniform_rng``, :443-460);
* the padded frame (``get_expanded_proj_2d_shape``, :516-562) and the zero
  padding (:651);
* the forward rotation by ``-180/pi * angle`` degrees (:667-679), the weight
  mask over the padded frame (:407-449, applied at :685-689) and the
  letterbox of detector columns (``get_letterbox_slice`` :462-492, applied at
  :690-749);
* Ram-Lak (and optionally Hilbert) linear convolution along u at pitch
  pixwid / L (:393-405; taps src/aprict/ramp_kernels.py:43-77);
* the rotation back by ``+180/pi * angle`` degrees (:790-806) and the crop
  (:836-842).

The rotations restate ``scipy.ndimage.rotate`` / ``affine_transform`` at
spline order 1 with mode "grid-constant" (reshape=False, prefilter=False):
output index o samples the input at ``M (o - c) + c`` with
``M = [[cos a, sin a], [-sin a, cos a]]`` and c the array centre, bilinear
weights, neighbours outside the array equal to 0. That is the published
definition implemented by ``cupyx.scipy.ndimage.rotate``, the call the
reference makes (cupy-cuda13x >= 14.2.0, a dependency not present under the
reference tree); the tests pin this restatement against
``scipy.ndimage.rotate`` itself. The angle chain follows that call: the
angle in degrees is a NumPy scalar of the angle array's dtype, converted with
``numpy.deg2rad`` and then ``math.cos`` / ``math.sin``.

``fbp_cone_cyl`` restates the reconstruction driver
(src/aprict/scripts/recon_cbfp_cyl_fbp.py:366-701, 1107-1238) with the FP64
backprojection oracle.
"""

from __future__ import annotations

import math

import numpy as np

# ---- taps (ramp_kernels.py:43-77) ----


def ramlak_taps(n: int, physpixsize: float) -> np.ndarray:
    """pi^2 (2 sinc(k) - sinc(k/2)^2) / physpixsize, k = -(n-1)/2 .. (n-1)/2 (ramp_kernels.py:43-59)."""
    k = np.arange(n, dtype=np.float64) - (n - 1) // 2
    return np.pi**2 * (2 * np.sinc(k) - np.sinc(k / 2) ** 2) / physpixsize


def hilbert_taps(n: int) -> np.ndarray:
    """2 / k, 0 at k = 0 (ramp_kernels.py:62-77)."""
    k = np.arange(n, dtype=np.float64) - (n - 1) // 2
    out = np.zeros(n)
    nz = k != 0
    out[nz] = 2.0 / k[nz]
    return out


def convolve_u(arr: np.ndarray, taps: np.ndarray) -> np.ndarray:
    """out[m, i, j] = sum_k taps[i - k + nu - 1] arr[m, k, j] (the zero-padded FFT convolution, :139-240)."""
    m, nu, nv = arr.shape
    out = np.empty(arr.shape, np.float64)
    for a in range(m):
        for j in range(nv):
            out[a, :, j] = np.convolve(arr[a, :, j].astype(np.float64), taps, mode="full")[nu - 1 : 2 * nu - 1]
    return out


# ---- geometry of the filter (ramp_filter.py:443-562) ----


def max_rotation_angle(nu: int, nv: int, physpixwid: float, L: float) -> float:  # noqa: N803
    """Half the vertical cone angle (:494-514)."""
    return float(np.arctan2(nv * physpixwid / 2, np.sqrt(np.square(L) + np.square(nu * physpixwid / 2))))


def expanded_shape(nu: int, nv: int, zeta: float, hacky: bool) -> tuple[int, int]:
    """The padded frame (:516-562)."""
    if hacky:
        return nu, nv
    w = int(np.ceil(nv * np.sin(zeta) + nu * np.cos(zeta)))
    h = int(np.ceil(nv))
    w += (w - nu) % 2
    h += (h - nv) % 2
    return w, h


def uniform_angles(rng: np.random.Generator, lo: float, hi: float, n: int) -> np.ndarray:
    """One rng.random() per element, stored as float32 (:443-460)."""
    out = np.empty((n,), dtype=np.float32)
    for i in range(n):
        out[i] = lo + (hi - lo) * rng.random()
    return out


def weight_mask(nu_e: int, nv_e: int, physpixwid: float, L: float, fdk: bool) -> np.ndarray:  # noqa: N803
    """Weights over the padded frame, with the reference's float32 grids (:407-449)."""
    u = physpixwid / L * (np.arange(nu_e, dtype=np.float32) - (nu_e - 1) / 2)
    v = physpixwid / L * (np.arange(nv_e, dtype=np.float32) - (nv_e - 1) / 2)
    if fdk:
        w = 1 / np.sqrt(1 + np.square(v[np.newaxis, :]) + np.square(u[:, np.newaxis]))
    else:
        w = 1 / (np.float_power(np.sqrt(1 + np.square(v[np.newaxis, :])), 3)
                 * np.sqrt(1 + np.square(v[np.newaxis, :]) + np.square(u[:, np.newaxis])))
    return np.asarray(w, dtype=np.float64)


def letterbox_columns(angle, zeta: float, L: float, physpixwid: float, nv_e: int) -> np.ndarray:  # noqa: N803
    """Per-column factor of the letterbox at one rotation angle (:462-492, :690-749)."""
    if abs(angle) > zeta:
        msg = "Invalid rotation angle entered."
        raise ValueError(msg)
    mid = (nv_e - 1) / 2
    disc = L / physpixwid * np.sqrt(np.maximum(np.square(np.cos(angle) / np.cos(zeta)) - 1, 0))
    start, stop = mid - disc, mid + disc
    i1, i2 = round(start), round(stop)
    w = np.ones(nv_e)
    if i1 == i2:
        w[i1] = stop - start
        w[:i1] = 0
        w[i1 + 1 :] = 0
    else:
        w[i1] = (i1 + 1 / 2) - start
        w[i2] = stop - (i2 - 1 / 2)
        w[:i1] = 0
        w[i2 + 1 :] = 0
    return w


def rotation_cs(angle_deg) -> tuple[float, float]:
    """(cos, sin) of a rotate() angle given in degrees, as the library call evaluates them."""
    rad = np.deg2rad(angle_deg)
    return math.cos(rad), math.sin(rad)


def rotate(img: np.ndarray, c: float, s: float, out_shape: tuple[int, int], centre: tuple[float, float],
           in_off: tuple[int, int] = (0, 0), out_off: tuple[int, int] = (0, 0)) -> np.ndarray:
    """Order-1 grid-constant resampling of a 2-D image placed at ``in_off`` in a
    frame with rotation centre ``centre``; output pixel (i, j) sits at
    ``(i, j) + out_off`` in the frame. FP64."""
    nu_in, nv_in = img.shape
    i = np.arange(out_shape[0], dtype=np.float64)[:, None] + out_off[0] - centre[0]
    j = np.arange(out_shape[1], dtype=np.float64)[None, :] + out_off[1] - centre[1]
    qu = (c * i + s * j + centre[0]) - in_off[0]
    qv = (-s * i + c * j + centre[1]) - in_off[1]
    fu, fv = np.floor(qu), np.floor(qv)
    tu, tv = qu - fu, qv - fv
    iu, iv = fu.astype(np.int64), fv.astype(np.int64)
    src = np.asarray(img, np.float64)

    def at(a, b):
        ok = (a >= 0) & (a < nu_in) & (b >= 0) & (b < nv_in)
        return np.where(ok, src[np.clip(a, 0, nu_in - 1), np.clip(b, 0, nv_in - 1)], 0.0)

    return (1 - tu) * ((1 - tv) * at(iu, iv) + tv * at(iu, iv + 1)) + tu * ((1 - tv) * at(iu + 1, iv) + tv * at(iu + 1, iv + 1))


# ---- the filter (ramp_filter.py:577-886) ----


def filter_tilted(arr: np.ndarray, *, L: float, physpixwid: float, angles: np.ndarray, zeta: float,  # noqa: N803
                  hilbert: bool = False, fan: bool = False, fdk: bool = False) -> list[np.ndarray]:
    """Filtered (M, nu, nv) arrays (ramp, then Hilbert if asked) for per-view rotation angles
    ``angles`` (the reference's angle array, float32 or float64). FP64 throughout, with the
    float32 roundings of the reference's intermediate arrays."""
    m, nu, nv = arr.shape
    hacky = fan or fdk
    nu_e, nv_e = expanded_shape(nu, nv, zeta, hacky)
    padx, pady = (nu_e - nu) // 2, (nv_e - nv) // 2
    centre = ((nu_e - 1) / 2, (nv_e - 1) / 2)
    mask = weight_mask(nu_e, nv_e, physpixwid, L, fdk)
    taps = [ramlak_taps(2 * nu_e - 1, physpixwid / L)] + ([hilbert_taps(2 * nu_e - 1)] if hilbert else [])
    outs = [np.zeros((m, nu, nv)) for _ in taps]
    for a in range(m):
        ang = angles[a]
        c, s = rotation_cs(-180 / np.pi * ang)
        e = rotate(arr[a], c, s, (nu_e, nv_e), centre, in_off=(padx, pady)).astype(np.float32)
        e = (e.astype(np.float64) * mask).astype(np.float32)
        if not hacky:
            e = (e.astype(np.float64) * letterbox_columns(ang, zeta, L, physpixwid, nv_e)[None, :]).astype(np.float32)
        cb, sb = rotation_cs(180 / np.pi * ang)
        for k, h in enumerate(taps):
            f = convolve_u(e[None], h)[0]
            outs[k][a] = rotate(f, cb, sb, (nu, nv), centre, out_off=(padx, pady))
    return outs


# ---- the driver (recon_cbfp_cyl_fbp.py:366-701, 1107-1238) ----


def fbp_cone_cyl(specs: np.ndarray, projs: np.ndarray, vol_shape: tuple[int, int, int], voxwid: float,
                 corner: np.ndarray, *, R: float, L: float, pixwid: float, zeta: float,  # noqa: N803
                 angles: np.ndarray, two_sided: bool, cyl_mask_rad: float, zs_span: float,
                 backproject) -> np.ndarray:
    """Cone-cylinder FBP with one rotation angle per projection (num_rot_angs None):
    filter, scale by 2 zeta / sin^2(zeta / 2), backproject with direct-raycast weights
    (preset 0 and (Z/R)^-3 one-sided; presets 1 and 6 with (Z/R)^-1 two-sided), scale the
    volume by (zs_max - zs_min) / (16 pi^2 R^2 M). ``backproject(specs, projs, cfg)`` is the
    backprojection oracle."""
    m = projs.shape[0]
    outs = filter_tilted(projs, L=L, physpixwid=pixwid, angles=angles, zeta=zeta, hilbert=two_sided)
    mult = 2 * zeta / np.float_power(np.sin(zeta / 2), 2)
    outs = [o * mult for o in outs]
    vol = np.zeros(vol_shape)
    if two_sided:
        cfgs = [dict(preset=1, pV=-1), dict(preset=6, pV=-1)]
    else:
        cfgs = [dict(preset=0, pV=-3)]
    for o, c in zip(outs, cfgs):
        vol += backproject(specs, o, dict(fast_approx=True, cyl_mask_rad=cyl_mask_rad, Z_on_val_factor_power=c["pV"],
                                          Z_on_val_factor_val=R, backproj_weighting_preset=c["preset"],
                                          approx_mode_direct_raycast=True))
    return vol * (zs_span / (16 * np.square(np.pi) * R**2 * m))
