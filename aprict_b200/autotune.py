"""Launch-shape autotuner.

Times a few candidate launch shapes of the forward projector (detector tile
height, warp patch shape, neighbouring views per tile) and the backprojector (voxels per thread, size of the brick-ordered
wave) on the caller's own problem with CUDA events, keeps the fastest, and
applies it through ``aprict_b200_set_tuning``. Results never depend on these
knobs; only speed does. Choices are cached per problem signature (in memory,
and optionally in a JSON file).
"""

from __future__ import annotations

import json
import pathlib
import threading

import torch

from . import _lib
from .cb import flatpanel as fp
from .volume import Volume

KEY_FP_TILE_V, KEY_BP_XB, KEY_BP_WAVE, KEY_FP_WARP_V, KEY_FP_VIEWS, KEY_FP_WARP_VIEWS, KEY_FP_SS1, KEY_BP_ZLANES = range(8)
FP_TILE_V = (8, 16, 32)
FP_WARP_V = (8, 16, 32)
FP_VIEWS = ((1, 1), (2, 1), (2, 2), (4, 1), (4, 2))  # (views per tile, views inside a warp)
BP_XB = (2, 4, 8)
BP_WAVE = (2, 3, 4, 6)

_cache: dict[str, dict] = {}
_lock = threading.Lock()


def _set(key: int, value: int) -> None:
    _lib.check(_lib.lib().aprict_b200_set_tuning(key, int(value)), "set_tuning")


def current() -> dict:
    """The knobs in effect (0 = built-in default)."""
    lib = _lib.lib()
    return {
        "fp_tile_v": lib.aprict_b200_get_tuning(KEY_FP_TILE_V),
        "fp_warp_v": lib.aprict_b200_get_tuning(KEY_FP_WARP_V),
        "fp_views": lib.aprict_b200_get_tuning(KEY_FP_VIEWS),
        "fp_warp_views": lib.aprict_b200_get_tuning(KEY_FP_WARP_VIEWS),
        "bp_xb": lib.aprict_b200_get_tuning(KEY_BP_XB),
        "bp_wave": lib.aprict_b200_get_tuning(KEY_BP_WAVE),
        "fp_ss1": lib.aprict_b200_get_tuning(KEY_FP_SS1),
        "bp_zlanes": lib.aprict_b200_get_tuning(KEY_BP_ZLANES),
    }


def apply(choice: dict) -> None:
    """Apply a choice returned by :func:`tune`."""
    _set(KEY_FP_TILE_V, choice.get("fp_tile_v", 0))
    _set(KEY_FP_WARP_V, choice.get("fp_warp_v", 0))
    _set(KEY_FP_VIEWS, choice.get("fp_views", 0))
    _set(KEY_FP_WARP_VIEWS, choice.get("fp_warp_views", 0))
    _set(KEY_BP_XB, choice.get("bp_xb", 0))
    _set(KEY_BP_WAVE, choice.get("bp_wave", 0))
    _set(KEY_FP_SS1, choice.get("fp_ss1", 0))
    _set(KEY_BP_ZLANES, choice.get("bp_zlanes", 0))


def _time(fn, reps: int = 3) -> float:
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def signature(projs: fp.ProjectionSet, volume: Volume, cfg_bp: fp.ConfigBackproject | None) -> str:
    """Cache key: data shapes, volume order and the backprojection settings."""
    c = None if cfg_bp is None else cfg_bp.contents.tobytes().hex()
    return json.dumps([list(projs.data.shape), list(volume.shape), volume.order, c])


def tune(
    projs: fp.ProjectionSet,
    volume: Volume,
    *,
    cfg_bp: fp.ConfigBackproject | None = None,
    multiplier: Volume | None = None,
    cache_file: str | pathlib.Path | None = None,
    reps: int = 2,
) -> dict:
    """Choose and apply the fastest launch shapes for this problem; returns the choice.

    Runs a handful of projections into a scratch copy of ``projs`` and
    backprojections into a scratch copy of ``volume``; the inputs are not modified.
    """
    sig = signature(projs, volume, cfg_bp)
    disk: dict = {}
    if cache_file is not None and pathlib.Path(cache_file).exists():
        disk = json.loads(pathlib.Path(cache_file).read_text())
    with _lock:
        if sig in _cache:
            apply(_cache[sig])
            return dict(_cache[sig])
        if sig in disk:
            _cache[sig] = disk[sig]
            apply(disk[sig])
            return dict(disk[sig])
    choice: dict = {}
    scratch_p = projs.zeroed_copy()
    cfg_fp = fp.ConfigProject()
    times = {}
    _set(KEY_FP_VIEWS, 1)
    _set(KEY_FP_WARP_VIEWS, 1)
    for tv in FP_TILE_V:
        for wv in FP_WARP_V:
            if wv > tv:
                continue
            _set(KEY_FP_TILE_V, tv)
            _set(KEY_FP_WARP_V, wv)
            times[(tv, wv)] = _time(lambda: fp.project(cfg_fp, volume, scratch_p), reps)
    best_fp = min(times, key=times.get)
    choice["fp_tile_v"], choice["fp_warp_v"] = best_fp
    _set(KEY_FP_TILE_V, best_fp[0])
    _set(KEY_FP_WARP_V, best_fp[1])
    vtimes = {(1, 1): times[best_fp]}
    for tw, ww in FP_VIEWS[1:]:
        _set(KEY_FP_VIEWS, tw)
        _set(KEY_FP_WARP_VIEWS, ww)
        vtimes[(tw, ww)] = _time(lambda: fp.project(cfg_fp, volume, scratch_p), reps)
    best_v = min(vtimes, key=vtimes.get)
    choice["fp_views"], choice["fp_warp_views"] = best_v
    choice["fp_ms"] = round(vtimes[best_v], 4)
    if cfg_bp is not None:
        scratch_v = volume.zeroed_copy()
        best = None
        for xb in BP_XB:
            for wave in BP_WAVE:
                _set(KEY_BP_XB, xb)
                _set(KEY_BP_WAVE, wave)
                t = _time(lambda: fp.backproject(cfg_bp, scratch_v, projs, summand_multiplier=multiplier), reps)
                if best is None or t < best[0]:
                    best = (t, xb, wave)
        choice["bp_xb"], choice["bp_wave"], choice["bp_ms"] = best[1], best[2], round(best[0], 4)
    apply(choice)
    with _lock:
        _cache[sig] = choice
        if cache_file is not None:
            disk[sig] = choice
            pathlib.Path(cache_file).write_text(json.dumps(disk, indent=1))
    return dict(choice)
