"""Analytic reconstruction drivers.

``fbp_fan_circ`` is the fan-beam FBP of the reference's ``aprict recon
fbp-fan-circ`` (src/aprict/scripts/cli.py:85-96 -> recon_cbfp_cyl_fbp.py with
fan_beam=True): per projection, weight by 1/sqrt(1 + u^2) and ramp-filter
with Ram-Lak taps at pitch pixwid/L (FBPFilterer, ramp_filter.py:343-449),
then backproject with direct-raycast weight (Z/R)^-2 (recon_cbfp_cyl_fbp.py:1108-1121;
CB_backproject.cu:512-528) inside the reconstructable cylinder, and scale by
1/(4 pi R M) (recon_cbfp_cyl_fbp.py:551-557).

Here the whole stack is filtered in one kernel launch with the weights and the
final scale folded in, then backprojected in one launch (the reference loops
over chunks of projections with several array passes each).

``fbp_cone_cyl`` is the cone-cylinder (helical) FBP of the same script
without the fan/FDK switches (recon_cbfp_cyl_fbp.py:366-701, 1107-1238):
tilted filtering (FBPFilterer with one random rotation angle per projection,
or the sum over ``num_rot_angs`` evenly spaced angles), the 2 zeta /
sin^2(zeta/2) normalisation, direct-raycast backprojection with weighting
preset 0 and (Z/R)^-3 (one-sided) or presets 1 and 6 with (Z/R)^-1 on the
ramp- and Hilbert-filtered data (two-sided), and the scale
(zs_max - zs_min) / (16 pi^2 R^2 M).

``gbc_cone_cyl`` is the GBC reconstruction of ``aprict recon gbc``
(src/aprict/scripts/recon_cbfp_cyl_gbc.py:371-1380): a padded volume and a
coarse (factor n) padded volume are backprojected with the GBC weights
(weighting preset 7) into the volume and its weight sums, scaled by
1/(mu R^2), the weight sums normalised by their expected value over a perfect
cylindrical locus, the volumes divided by the soft-zeroed weight sums, the
coarse volume filtered padded and unpadded to form a low-frequency
correction, the volume filtered with that correction added, its DC level
estimated on the boundary and subtracted, and the padding cropped.
"""

from __future__ import annotations

import numpy as np
import torch

import math

from .cb import flatpanel as fp
from .cb.ramp_filter import FBPFilterer
from .volume import Volume


def fan_geometry(pg: fp.ProjGeom) -> tuple[float, float, float, int, int]:
    """(R, L, pixwid, nu, nv) of a circular scan, with the reference's checks (recon_cbfp_cyl_fbp.py:459-496)."""
    if len(pg.projs_list_shape) != 1:
        msg = f"Input projection geometry has a non-flat shape: {pg.projs_list_shape}."
        raise NotImplementedError(msg)
    nus, nvs = np.broadcast_to(pg.nu, pg.projs_list_shape), np.broadcast_to(pg.nv, pg.projs_list_shape)
    if not (np.all(nus == nus[0]) and np.all(nvs == nvs[0])):
        msg = "Inconsistent detector resolution."
        raise NotImplementedError(msg)
    pixwids = np.linalg.norm(np.broadcast_to(pg.det_uvec, pg.projs_list_shape + (3,)), axis=-1)
    pixheis = np.linalg.norm(np.broadcast_to(pg.det_vvec, pg.projs_list_shape + (3,)), axis=-1)
    if not (np.allclose(pixwids, pixwids[0]) and np.allclose(pixheis, pixheis[0]) and np.isclose(pixwids[0], pixheis[0])):
        msg = "Inconsistent or non-square detector pixels."
        raise NotImplementedError(msg)
    src = np.broadcast_to(pg.source_pos, pg.projs_list_shape + (3,)).astype(np.float64)
    det = np.broadcast_to(pg.det_pos, pg.projs_list_shape + (3,)).astype(np.float64)
    Rs = np.hypot(src[:, 0], src[:, 1])  # noqa: N806
    if not np.allclose(Rs, Rs[0]):
        msg = "Inconsistent source radius."
        raise NotImplementedError(msg)
    Ls = Rs + np.hypot(det[:, 0], det[:, 1])  # noqa: N806
    if not np.allclose(Ls, Ls[0]):
        msg = "Inconsistent source-to-detector length."
        raise NotImplementedError(msg)
    return float(Rs[0]), float(Ls[0]), float(pixwids[0]), int(nus[0]), int(nvs[0])


def fbp_fan_circ(
    projs: fp.ProjectionSet,
    volume: Volume,
    *,
    interpolate: bool = False,
    apodization: str | None = None,
    cyl_mask_rad: float | None = None,
    filtered_out: torch.Tensor | None = None,
) -> Volume:
    """Add the fan-beam FBP reconstruction of ``projs`` (M, nu, 1) into ``volume``."""
    if projs.data is None:
        msg = "You must provide projection data."
        raise ValueError(msg)
    R, L, pixwid, nu, nv = fan_geometry(projs.proj_geom)  # noqa: N806
    m = projs.proj_geom.num_projs
    filt = FBPFilterer(L=L, physpixwid=pixwid, proj_2d_shape=(nu, nv), _hacky_fan_beam_mode=True, apodization=apodization)
    scale = 1.0 / (4.0 * np.pi * R * m)
    outs = None if filtered_out is None else [filtered_out]
    (filtered,) = filt.rfilt.filter(projs.data.float(), weights=filt._weights, scale=scale, outs=outs)  # noqa: SLF001
    support = R * np.sin(np.arctan(pixwid * nu / 2 / L))
    cfg = fp.ConfigBackproject(
        fast_approx=True,
        cyl_mask_rad=cyl_mask_rad or support,
        Z_on_val_factor_power=-2,
        Z_on_val_factor_val=R,
        approx_mode_direct_raycast=True,
        approx_mode_bilinear_interpolate=interpolate,
    )
    fp.backproject(cfg, volume, fp.ProjectionSet(projs.proj_geom, data=filtered))
    return volume


def fbp_fan_circ_batch(
    projs: list[fp.ProjectionSet],
    volumes: list[Volume],
    *,
    apodization: str | None = None,
    interpolate: bool = False,
    stacked: torch.Tensor | None = None,
) -> list[Volume]:
    """Fan-beam FBP of many slices (each a scan with nv = 1) in two launches.

    Every slice must share the fan geometry (R, L, pixel pitch, nu) and view
    count, as the slices of one fan-beam stack do; then one ramp-filter launch
    filters all sinograms (``stacked``: an (S*M, nu, 1) tensor holding them,
    filtered in place into a new buffer; assembled from ``projs`` if None) and
    one persistent backprojection launch (:class:`~aprict_b200.batch.ScanBatch`)
    backprojects every slice into its volume. Each slice's result equals
    :func:`fbp_fan_circ` on that slice.
    """
    from .batch import ScanBatch  # noqa: PLC0415

    if not projs or len(projs) != len(volumes):
        msg = "one volume per sinogram, at least one"
        raise ValueError(msg)
    # slices of one stack usually share one ProjGeom object: check each distinct one once
    by_id: dict[int, tuple] = {}
    for p in projs:
        if id(p.proj_geom) not in by_id:
            by_id[id(p.proj_geom)] = fan_geometry(p.proj_geom)
    geo = [by_id[id(p.proj_geom)] for p in projs]
    m = projs[0].proj_geom.num_projs
    if any(not np.allclose(g, geo[0]) for g in geo) or any(p.proj_geom.num_projs != m for p in projs):
        msg = "batched fan FBP needs one fan geometry and view count for every slice"
        raise NotImplementedError(msg)
    R, L, pixwid, nu, nv = geo[0]  # noqa: N806
    if stacked is None:
        stacked = torch.cat([p.data.float() for p in projs], dim=0)
    filt = FBPFilterer(L=L, physpixwid=pixwid, proj_2d_shape=(nu, nv), _hacky_fan_beam_mode=True, apodization=apodization)
    (filtered,) = filt.rfilt.filter(stacked, weights=filt._weights, scale=1.0 / (4.0 * np.pi * R * m))  # noqa: SLF001
    support = R * np.sin(np.arctan(pixwid * nu / 2 / L))
    cfg = fp.ConfigBackproject(
        fast_approx=True, cyl_mask_rad=support, Z_on_val_factor_power=-2, Z_on_val_factor_val=R,
        approx_mode_direct_raycast=True, approx_mode_bilinear_interpolate=interpolate,
    )
    views = [p._with_data(filtered[i * m : (i + 1) * m]) for i, p in enumerate(projs)]  # noqa: SLF001
    ScanBatch(volumes, views).backproject(cfg)
    return volumes


def fbp_cone_cyl(
    projs: fp.ProjectionSet,
    volume: Volume,
    *,
    two_sided: bool = False,
    num_rot_angs: int | None = None,
    limit_zeta: float | None = None,
    seed_proj_rots: int | None = None,
    interpolate: bool = False,
    ssx: int = 1,
    ssy: int = 1,
    ssz: int = 1,
    cyl_mask_rad: float | None = None,
    num_projs_per_chunk: int = 64,
) -> Volume:
    """Add the cone-cylinder FBP reconstruction of ``projs`` (M, nu, nv) into ``volume``.

    Projections are filtered and backprojected ``num_projs_per_chunk`` at a
    time; a chunk whose sources lie entirely out of reach of the volume along
    z is skipped (its rotation angles are still drawn), as in the reference
    (recon_cbfp_cyl_fbp.py:565-607).
    """
    if projs.data is None:
        msg = "You must provide projection data."
        raise ValueError(msg)
    if num_projs_per_chunk <= 0:
        msg = "num_projs_per_chunk must be positive"
        raise ValueError(msg)
    pg = projs.proj_geom
    R, L, pixwid, nu, nv = fan_geometry(pg)  # noqa: N806
    m = pg.num_projs
    src_z = np.broadcast_to(pg.source_pos, pg.projs_list_shape + (3,))[:, 2].astype(np.float64)
    zs_max, zs_min = float(src_z.max()), float(src_z.min())
    vartheta_v = np.arctan2(nv * pixwid / 2 - pixwid / 2, np.sqrt(np.square(L) + np.square(nu * pixwid / 2 - pixwid / 2)))
    support = R * np.sin(np.arctan(pixwid * nu / 2 / L))
    cyl_mask_rad = cyl_mask_rad or support
    (x0, y0, z0), (x1, y1, z1) = volume.minxyz_maxxyz
    max_r = min(cyl_mask_rad, float(np.sqrt(max(abs(x0), abs(x1)) ** 2 + max(abs(y0), abs(y1)) ** 2)))
    vartheta_eff = min(limit_zeta, vartheta_v) if limit_zeta is not None else vartheta_v
    hdiff = np.tan(vartheta_eff) * (R + max_r)
    filt = FBPFilterer(
        proj_2d_shape=(nu, nv), projs_per_batch=num_projs_per_chunk, L=L, physpixwid=pixwid, limit_zeta=limit_zeta,
        include_hilbert_transform_in_output=two_sided, rng=np.random.default_rng(seed=seed_proj_rots),
    )
    zeta = filt.zeta
    if num_rot_angs is None:
        angs = None
    elif num_rot_angs == 1:
        angs = np.array([0.0], dtype=np.float32)
    else:
        angs = np.linspace(-zeta + (2 * zeta / num_rot_angs / 2), zeta - (2 * zeta / num_rot_angs / 2), endpoint=True,
                           num=num_rot_angs)
    norm = 2 * zeta / np.float_power(np.sin(zeta / 2), 2) / (1 if angs is None else len(angs))
    scale = float(norm * (zs_max - zs_min) / (16 * np.square(np.pi) * R**2 * m))
    common = dict(fast_approx=True, cyl_mask_rad=cyl_mask_rad, Z_on_val_factor_val=R, approx_mode_direct_raycast=True,
                  approx_mode_bilinear_interpolate=interpolate, ssx=ssx, ssy=ssy, ssz=ssz)
    if two_sided:
        cfgs = [fp.ConfigBackproject(Z_on_val_factor_power=-1, backproj_weighting_preset=1, **common),
                fp.ConfigBackproject(Z_on_val_factor_power=-1, backproj_weighting_preset=6, **common)]
    else:
        cfgs = [fp.ConfigBackproject(Z_on_val_factor_power=-3, backproj_weighting_preset=0, **common)]
    data = projs.data
    for a in range(0, m, num_projs_per_chunk):
        sl = slice(a, min(m, a + num_projs_per_chunk))
        if z1 < src_z[sl].min() - hdiff or z0 > src_z[sl].max() + hdiff:
            filt.advance_rng(sl.stop - sl.start)  # out of reach of the volume
            continue
        chunk = data[sl].float()
        if angs is None:
            outs, _ = filt.filter_bulk_axis1_concat(chunk, force_rotation_angle=None, block=False)
        else:
            outs = None
            for ang in angs:
                o, _ = filt.filter_bulk_axis1_concat(chunk, force_rotation_angle=ang, block=False)
                outs = o if outs is None else [x.add_(y) for x, y in zip(outs, o)]
        for o, cfg in zip(outs, cfgs):
            o.mul_(scale)
            fp.backproject(cfg, volume, fp.ProjectionSet(pg.sliced(sl), data=o))
    return volume


def gbc_cone_cyl(
    projs: fp.ProjectionSet,
    volshape: tuple[int, int, int],
    voxwid: float,
    volpos: tuple[float, float, float] = (0.0, 0.0, 0.0),
    *,
    n: int = 9,
    f1: float = 1.2,
    f2: float = 6.0,
    eps: float = 1e-6,
    softspan_v: float = 0.05,
    softspan_h: float = 0.05,
    interpolate_measurements: bool = True,
    ssx: int = 1,
    ssy: int = 1,
    ssz: int = 1,
    num_projs_per_chunk: int = 64,
    num_z_samps: int = 6000,
    num_ang_samps: int = 6000,
) -> Volume:
    """GBC reconstruction of ``projs`` (M, nu, nv) from a cylindrical source
    locus into a new (``volshape``, ``voxwid``, ``volpos``) volume.

    Options follow the reference's CLI (recon_cbfp_cyl_gbc.py:166-240): ``n``
    (odd) the coarse volume's downscale factor, ``f1`` / ``f2`` the padding
    factors of the full and coarse volumes, ``eps`` the soft-zero of the
    weight division, ``softspan_v`` / ``softspan_h`` the soft window spans.
    The reference processes the volumes in z slabs to fit device memory;
    here each volume is one array (the result is the same: every step is
    per voxel, and the filters act on the whole arrays in both).
    """
    from .gbc import filters, weightinteg  # noqa: PLC0415

    if projs.data is None:
        msg = "You must provide projection data."
        raise ValueError(msg)
    if n < 1 or n % 2 == 0:
        msg = "n must be a positive odd integer."
        raise ValueError(msg)
    if min(ssx, ssy, ssz) <= 0:
        msg = "ssx, ssy, ssz must all be positive integers."
        raise ValueError(msg)
    volshape = tuple(int(s) for s in volshape)
    # padded shapes (recon_cbfp_cyl_gbc.py:649-684)
    padded = tuple(n * (4 + math.ceil(s * f1 / n)) for s in volshape)
    padded = tuple(p if (p - s) % 2 == 0 else p + n for s, p in zip(volshape, padded))
    pads = tuple((p - s) // 2 for s, p in zip(volshape, padded))
    mini = tuple(math.ceil(s * f2 / n) for s in volshape)
    mini = tuple(max(m, p // n) for p, m in zip(padded, mini))
    mini = tuple(m if (m - p // n) % 2 == 0 else m + 1 for p, m in zip(padded, mini))
    mpads = tuple((m - p // n) // 2 for p, m in zip(padded, mini))

    vol = Volume.zeros(padded, voxwid=voxwid, pos_c=volpos)
    vol_ws = Volume.zeros(padded, voxwid=voxwid, pos_c=volpos)
    minivol = Volume.zeros(mini, voxwid=voxwid * n, pos_c=volpos)
    minivol_ws = Volume.zeros(mini, voxwid=voxwid * n, pos_c=volpos)

    # geometry (recon_cbfp_cyl_gbc.py:371-534)
    pg = projs.proj_geom
    R, L, pixwid, nu, nv = fan_geometry(pg)  # noqa: N806
    m = pg.num_projs
    vartheta_v = float(np.arctan2(nv * pixwid / 2 - pixwid / 2, np.sqrt(L**2 + (nu * pixwid / 2 - pixwid / 2) ** 2)))
    vartheta_h = float(np.arctan2(nu * pixwid / 2 - pixwid / 2, L))
    src_z = np.broadcast_to(pg.source_pos, pg.projs_list_shape + (3,))[:, 2].astype(np.float64)
    zs_max, zs_min = float(src_z.max()), float(src_z.min())
    (x0, y0, z0), (x1, y1, z1) = minivol.minxyz_maxxyz
    max_r = float(np.sqrt(max(abs(x0), abs(x1)) ** 2 + max(abs(y0), abs(y1)) ** 2))
    hdiff = np.tan(vartheta_v) * (R + max_r)
    mu = m / (2 * np.pi * R * (zs_max - zs_min))
    cfg = fp.ConfigBackproject(
        fast_approx=True, Z_on_val_factor_val=R, backproj_weighting_preset=7, approx_mode_direct_raycast=True,
        approx_mode_bilinear_interpolate=interpolate_measurements, ssx=ssx, ssy=ssy, ssz=ssz,
        soft_vartheta_v=vartheta_v, soft_vartheta_v_softspan=softspan_v, soft_vartheta_h=vartheta_h,
        soft_vartheta_h_softspan=softspan_h,
    )

    def divisor(v: Volume) -> np.ndarray:
        xs, ys, _ = v.xs_ys_zs
        integ = weightinteg.backproj_gbc_weight_integ_xygrid_GPU(xs, ys, R, cfg, num_z_samps, num_ang_samps)
        return np.power(integ, -1).astype(np.float32)

    div_full, div_mini = divisor(vol), divisor(minivol)

    # backprojection of every chunk of views within reach of the volumes (:1104-1190)
    done = 0
    for a in range(0, m, num_projs_per_chunk):
        sl = slice(a, min(m, a + num_projs_per_chunk))
        if z1 < src_z[sl].min() - hdiff or z0 > src_z[sl].max() + hdiff:
            continue
        ps = fp.ProjectionSet(pg.sliced(sl), data=projs.data[sl])
        fp.backproject(cfg, vol, ps, secondary_volume=vol_ws)
        fp.backproject(cfg, minivol, ps, secondary_volume=minivol_ws)
        done += sl.stop - sl.start
    if done > 0:  # (:1191-1222)
        factor = 1 / (mu * R**2)
        for v in (vol, vol_ws, minivol, minivol_ws):
            v.multiply(factor)
        vol_ws.multiply_by_xygrid(div_full)
        minivol_ws.multiply_by_xygrid(div_mini)
        vol.divide_softzero(vol_ws, eps=eps)
        minivol.divide_softzero(minivol_ws, eps=eps)
    del vol_ws, minivol_ws

    # filtering with the low-frequency correction (:1245-1324)
    cone = 2 * vartheta_v
    crop_m = tuple(slice(p, (-p) or None) for p in mpads)
    mini_pad_f = filters.ramp_filter_conebeam(minivol.data, voxwid * n, cone, theta_soft=softspan_v)
    mini_unpad_f = filters.ramp_filter_conebeam(minivol.data[crop_m].contiguous(), voxwid * n, cone,
                                                theta_soft=softspan_v)
    correction = mini_pad_f[crop_m] - mini_unpad_f
    del mini_pad_f, mini_unpad_f, minivol
    out = filters.ramp_filter_conebeam(vol.data, voxwid, cone, theta_soft=softspan_v,
                                       lowres_correction_array=correction.contiguous())
    del vol, correction
    # DC level from the boundary of the central region (:1326-1352)
    c = out[2 * n : -2 * n, 2 * n : -2 * n, 2 * n : -2 * n]
    dc = 0.25 * (c[:, 0, :].double().mean() + c[:, -1, :].double().mean() + c[0, :, :].double().mean()
                 + c[-1, :, :].double().mean())
    out -= dc.float()
    crop = tuple(slice(p, (-p) or None) for p in pads)
    res = Volume.zeros(volshape, voxwid=voxwid, pos_c=volpos)
    res.data.copy_(out[crop])
    return res
