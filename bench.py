"""Benchmark: SIRT iterations/s (with forward rays/s and back voxel-updates/s) on one B200.

Workload (default ``sirt256``): a 256^3 float32 volume (0.5 mm voxels) of 30
seeded random ellipsoids, a circular cone-beam scan of 360 views on a 384x384
flat detector (0.8 mm pixels, SOD 500 mm, SDD 1000 mm), and the reference's
SIRT iteration x <- x + M (.) B (b - A x) (src/aprict/iterators/sirt_vram.py:130-152):
A the exact Siddon projector, B the fast backprojector with cylinder mask and
5 % detector-edge taper, M the preconditioner. The data b are synthetic
(A x_true + Poisson noise at 1e5 photons); nothing is read from disk.

A step is one SIRT iteration. ``value`` is the batched form (fused residual +
one all-view backprojection, replayed from a captured CUDA graph); the
plain-launch form of the same kernels (copy, atomic projection, 10-view
backprojection launches with host synchronisation -- the reference's launch
pattern) is reported beside it. The inputs (b 202 MB, residual 202 MB, x and
M 64 MB each) exceed the 126 MB L2, so no flush is needed between steps.

``--impl reference`` times the reference's own device code compiled for the CPU
(oracle/_ref), on a bounded sample of the same iteration scaled to iter/s.
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SIRT iter/s"
HEADLINE_METRIC = "fwd rays/s, back voxel-updates/s, SIRT iter/s: batched vs plain at rel L2 1e-5"

WORKLOADS = {
    "sirt256": dict(
        n=256, voxwid=0.5, n_ellipsoids=30, views=360, det=384, pix_at_iso=0.4, R=500.0, LmR=500.0, photons=1e5,
        seed=4,
    ),
    "small": dict(n=96, voxwid=1.0, n_ellipsoids=10, views=90, det=128, pix_at_iso=0.8, R=300.0, LmR=300.0, photons=1e5, seed=1),
    # 48 uneven scans: edge log-U(64, 320), views U(90, 720), detector U(128, 768)^2,
    # circular or helical (pitch U(0.5, 1.5)), +-2 mm / +-0.5 deg per-view jitter.
    # Component workloads (each prints its own line):
    # fpbp128 -- 128^3 x 1 mm, 10 ellipsoids, 180 views on 256^2 x 1 mm, SOD 500, SDD 1000;
    # fbp64 -- 64 fan-beam slices 512^2 x 0.5 mm, 720 views, 1024 x 0.4 mm, SOD 600, SDD 1100;
    # quadric -- 100 clipped quadrics (60 ellipsoids, 40 elliptic cylinders) in 200 mm,
    #   720 views on 1024^2 x 0.3 mm, SOD 700, SDD 1200, additive densities.
    "fpbp128": dict(n=128, voxwid=1.0, n_ellipsoids=10, views=180, det=256, pix_at_iso=0.5, R=500.0, LmR=500.0, seed=3),
    "fbp64": dict(slices=64, n=512, voxwid=0.5, n_ellipses=20, views=720, det=1024, pix=0.4, R=600.0, LmR=500.0, seed=7),
    # fbpcyl -- cone-cylinder FBP: 256^3 x 0.5 mm, 720 golden-angle views on a 500 mm cylinder
    #   (80 mm high) x 384^2 x 0.8 mm, tilted filtering + direct-raycast backprojection;
    # gbc -- GBC reconstruction: 128^3 x 1 mm, 360 views on a 500 mm cylinder (128 mm high)
    #   x 256^2 x 1.5 mm, n = 9, f1 = 1.2, f2 = 6, 6000 x 6000 weight-integral samples.
    "fbpcyl": dict(n=256, voxwid=0.5, n_ellipsoids=30, views=720, det=384, pix_at_iso=0.4, R=500.0, LmR=500.0,
                   height=80.0, seed=11),
    "gbc": dict(n=128, voxwid=1.0, n_ellipsoids=20, views=360, det=256, pix_at_iso=0.75, R=500.0, LmR=500.0,
                height=128.0, seed=12),
    "quadric": dict(n_ellipsoids=60, n_cylinders=40, radius=100.0, views=720, det=1024, pix=0.3, R=700.0, LmR=500.0,
                    seed=11),
    "batch48": dict(n_scans=48, edge=(64, 320), views=(90, 720), det=(128, 768), voxwid=0.5, n_ellipsoids=10,
                    R=500.0, LmR=500.0, photons=1e5, seed=5),
}


def _env_rank() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def make_problem(w: dict):
    from aprict_b200 import phantoms
    from aprict_b200.cb import flatpanel as fp

    n = w["n"]
    pg = fp.ProjGeom.new_circular_scan(
        num_source_points=w["views"], R=w["R"], L_minus_R=w["LmR"], pix_widhei_at_isocenter=(w["pix_at_iso"],) * 2,
        num_pix_widhei=(w["det"], w["det"]),
    )
    x_true = phantoms.ellipsoid_volume(w["seed"], w["n_ellipsoids"], (n, n, n), w["voxwid"], semi_axes_vox=(10, 80 * n / 256))
    return pg, x_true


def simulate_data(pg, x_true: np.ndarray, w: dict):
    """b = -log(Poisson(I0 exp(-A x))/I0), capped at log I0 (examples/fan_beam_sirt.py:156-180)."""
    import torch

    from aprict_b200 import Volume
    from aprict_b200.cb import flatpanel as fp

    v = Volume(x_true, voxwid=w["voxwid"])
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), v, ps, block=True)
    g = torch.Generator(device="cuda").manual_seed(w["seed"])
    lam = w["photons"] * torch.exp(-ps.data.double())
    counts = torch.poisson(lam, generator=g).clamp_(min=1.0)
    b = (-torch.log(counts / w["photons"])).clamp_(max=float(np.log(w["photons"]))).float()
    return b


class ClockSampler:
    """Samples nvidia-smi clocks during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index: int) -> None:
        self.gpu = gpu_index
        self.proc = None
        self.path = pathlib.Path(tempfile.mkstemp(suffix=".csv")[1])

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")  # noqa: SIM115
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL,
            )
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self) -> dict | None:
        if self.proc is None or not self.path.exists():
            return None
        rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, val in zip(names, r[5:9]):
                if "Active" in val and "Not" not in val:
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons),
            "samples": len(rows),
        }


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic() -> dict:
    p = ROOT / "profiles" / "traffic.json"
    return json.loads(p.read_text()) if p.exists() else {}


def count_segments(pg, x_shape, voxwid: float, sample_views: int = 4) -> tuple[float, int]:
    """Sum of ray/voxel segments over the whole scan, from the FP64 oracle on a view sample.

    Circular scans are rotationally equivalent up to the volume's cubic
    symmetry, so the per-view count of evenly spaced sample views scales.
    """
    from oracle import oracle

    m = pg.num_projs
    idx = list(np.linspace(0, m, sample_views, endpoint=False).astype(int))
    specs = pg.to_proj_spec_array()[idx]
    ones = np.ones(x_shape, np.float32)
    corner = -np.float32(voxwid) * np.array(x_shape, np.float32) / 2
    _, nseg = oracle.project_siddon(specs, ones, voxwid=voxwid, corner=corner)
    return nseg * m / sample_views, nseg


def run_ours(args) -> dict:
    import torch

    from aprict_b200 import Volume
    from aprict_b200.cb import flatpanel as fp
    from aprict_b200.iterators import SIRT_flatpanel

    from aprict_b200 import replicas

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    replicas.init("nccl")
    w = WORKLOADS[args.workload]
    if args.workload == "gbc":  # per step: one GBC backprojection of the padded volume, one weight integral
        from aprict_b200 import geometry
        from aprict_b200.gbc import weightinteg

        n, m, vw = w["n"], w["views"], w["voxwid"]
        pg = geometry.cylinder_scan(n_views=m, R=w["R"], L_minus_R=w["LmR"], pix_at_iso=w["pix_at_iso"],
                                    nu=w["det"], nv=w["det"], height=w["height"])
        gen = torch.Generator(device="cuda")
        gen.manual_seed(w["seed"])
        ps = fp.ProjectionSet(pg, data=torch.rand((m, w["det"], w["det"]), device="cuda", generator=gen))
        L = w["R"] + w["LmR"]  # noqa: N806
        pixwid = float(np.linalg.norm(pg.det_uvec[0]))
        nu = nv = w["det"]
        cfg = fp.ConfigBackproject(
            fast_approx=True, Z_on_val_factor_val=w["R"], backproj_weighting_preset=7, approx_mode_direct_raycast=True,
            approx_mode_bilinear_interpolate=True,
            soft_vartheta_v=float(np.arctan2(nv * pixwid / 2 - pixwid / 2, np.sqrt(L**2 + (nu * pixwid / 2 - pixwid / 2) ** 2))),
            soft_vartheta_v_softspan=0.05, soft_vartheta_h=float(np.arctan2(nu * pixwid / 2 - pixwid / 2, L)),
            soft_vartheta_h_softspan=0.05)
        pad = 9 * (4 + int(np.ceil(n * 1.2 / 9)))
        pad = pad if (pad - n) % 2 == 0 else pad + 9
        vol, ws = Volume.zeros((pad,) * 3, voxwid=vw), Volume.zeros((pad,) * 3, voxwid=vw)
        xs = vol.xs_ys_zs[0]
        for _ in range(args.steps):
            fp.backproject(cfg, vol, ps, secondary_volume=ws)
            weightinteg.backproj_gbc_weight_integ_xygrid_GPU(xs, xs, w["R"], cfg)
        torch.cuda.synchronize()
        return {"mode": "kernels", "workload": args.workload, "launches": 2 * args.steps}
    if args.workload == "fbpcyl":  # one direct-raycast backprojection of the cone-cylinder FBP per step
        from aprict_b200 import geometry

        n, m = w["n"], w["views"]
        pg = geometry.cylinder_scan(n_views=m, R=w["R"], L_minus_R=w["LmR"], pix_at_iso=w["pix_at_iso"],
                                    nu=w["det"], nv=w["det"], height=w["height"])
        gen = torch.Generator(device="cuda")
        gen.manual_seed(w["seed"])
        ps = fp.ProjectionSet(pg, data=torch.rand((m, w["det"], w["det"]), device="cuda", generator=gen))
        L = w["R"] + w["LmR"]  # noqa: N806
        pixwid = float(np.linalg.norm(pg.det_uvec[0]))
        cfg = fp.ConfigBackproject(fast_approx=True, cyl_mask_rad=w["R"] * np.sin(np.arctan(pixwid * w["det"] / 2 / L)),
                                   Z_on_val_factor_power=-3, Z_on_val_factor_val=w["R"], approx_mode_direct_raycast=True)
        out = Volume.zeros((n, n, n), voxwid=w["voxwid"])
        for _ in range(args.steps):
            fp.backproject(cfg, out, ps)
        torch.cuda.synchronize()
        return {"mode": "kernels", "workload": args.workload, "launches": args.steps}
    n = w["n"]
    pg, x_true = make_problem(w)
    b = simulate_data(pg, x_true, w)
    meas = fp.ProjectionSet(pg, data=b)
    x = Volume.zeros((n, n, n), voxwid=w["voxwid"])
    sirt = SIRT_flatpanel(SIRT_flatpanel.Config(), x, meas)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()

    barrier = replicas.barrier
    max_over_ranks = replicas.max_over_ranks

    # ---- component kernels (CUDA events on the launching stream) ----
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    def time_op(fn, reps: int) -> float:
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        s, e = ev(), ev()
        s.record(stream)
        for _ in range(reps):
            fn()
        e.record(stream)
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    cfg_res = fp.ConfigProject(multiply_before_adding=-1)
    r = sirt._scratch  # noqa: SLF001
    t_fp = time_op(lambda: fp.project_residual(cfg_res, x, r, meas.data), 3)
    t_bp = time_op(lambda: fp.backproject(sirt._config_bp, x, r, summand_multiplier=sirt.preconditioner), 3)  # noqa: SLF001
    x.fill(0.0)

    # ---- batched: graph-captured iterations ----
    sirt.iterate_graph(1)  # warm-up + capture (1 iteration per replay)
    sirt.iterate_graph(1)
    for _ in range(max(0, args.warmup - 2)):
        sirt.iterate_graph(1)
    barrier()
    with ClockSampler(local) as clk:
        s, e = ev(), ev()
        s.record(stream)
        for _ in range(args.steps):
            sirt.iterate_graph(1)
        e.record(stream)
        torch.cuda.synchronize()
        ms = s.elapsed_time(e) / args.steps
    ms = max_over_ranks(ms)
    barrier()

    # ---- plain launches: the reference's pattern with the same kernels ----
    chunks = []
    for c0 in range(0, pg.num_projs, 10):
        sl = slice(c0, min(c0 + 10, pg.num_projs))
        chunks.append(fp.ProjectionSet(pg.sliced(sl), data=r.data[sl]))
    cfg_acc = fp.ConfigProject(multiply_before_adding=-1)

    def plain_iter() -> None:
        r.data.copy_(meas.data)
        fp.project(cfg_acc, x, r, block=True)
        for ch in chunks:
            fp.backproject(sirt._config_bp, x, ch, summand_multiplier=sirt.preconditioner)  # noqa: SLF001
        torch.cuda.synchronize()

    for _ in range(2):
        plain_iter()
    barrier()
    t0 = time.perf_counter()
    s, e = ev(), ev()
    s.record(stream)
    k_plain = max(3, args.steps // 2)
    for _ in range(k_plain):
        plain_iter()
    e.record(stream)
    torch.cuda.synchronize()
    ms_plain = max_over_ranks(s.elapsed_time(e) / k_plain)

    # ---- end to end through the public API with host buffers ----
    b_host = b.cpu().pin_memory()
    x_host = torch.empty((n, n, n), dtype=torch.float32).pin_memory()
    def e2e_iter() -> None:
        sirt.iterate_from_host(b_host, x_host)

    for _ in range(2):
        e2e_iter()
    sirt.host_sync()
    barrier()
    s, e = ev(), ev()
    s.record(stream)
    for _ in range(args.steps):
        e2e_iter()
    stream.wait_stream(sirt._pipe.up)  # noqa: SLF001  the last transfers end inside the timed region
    stream.wait_stream(sirt._pipe.down)  # noqa: SLF001
    e.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(s.elapsed_time(e) / args.steps)

    # ---- accounting ----
    M = pg.num_projs
    rays = M * w["det"] ** 2
    vox = n**3
    nseg, nseg_sample = count_segments(pg, (n, n, n), w["voxwid"])
    fp_bytes = 4.0 * nseg + 8.0 * rays  # one gather per segment; read b, write r
    bp_bytes = 4.0 * vox * M + 12.0 * vox  # one detector sample per voxel-view; read M, RMW x
    peak, peak_kind = load_peaks()
    fp_gbs = fp_bytes / (t_fp * 1e-3) / 1e9
    bp_gbs = bp_bytes / (t_bp * 1e-3) / 1e9
    dom = "project_siddon" if t_fp >= t_bp else "backproject"
    tr = load_traffic().get(f"{dom}:{args.workload}")
    traffic = tr["dram_bytes"] if tr else None
    roof = {
        "bound": "hbm",
        "kernel": dom,
        "achieved": round(fp_gbs if dom == "project_siddon" else bp_gbs, 1),
        "peak": peak,
        "unit": "GB/s",
        "frac": round((fp_gbs if dom == "project_siddon" else bp_gbs) / peak, 4),
        "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s",
        "traffic": traffic,
        "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/)",
        "algorithmic_bytes": round(fp_bytes if dom == "project_siddon" else bp_bytes),
        "model": "FP: 4 B per ray/voxel segment + 8 B per ray; BP: 4 B per voxel-view + 12 B per voxel",
    }
    out = {
        "metric": METRIC,
        "value": round(world * 1000.0 / ms, 4),
        "unit": "iter/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded ellipsoid phantom, simulated Poisson data)",
        "config": {
            "workload": workload_text(args.workload, w, M),
            "baseline_metric": HEADLINE_METRIC,
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "l2": "inputs larger than L2 (b+r 404 MB, x+M 128 MB)",
            "form": "batched: fused residual + all-view backprojection, CUDA-graph replay",
        },
        "components": {
            "fwd_rays_per_s": round(rays / (t_fp * 1e-3), 1),
            "fwd_ray_steps_per_s": round(nseg / (t_fp * 1e-3), 1),
            "back_voxel_updates_per_s": round(vox * M / (t_bp * 1e-3), 1),
            "fp_ms": round(t_fp, 4),
            "bp_ms": round(t_bp, 4),
            "fp_GBps": round(fp_gbs, 1),
            "bp_GBps": round(bp_gbs, 1),
            "segments_per_scan": nseg,
            "plain_iter_per_s": round(world * 1000.0 / ms_plain, 4),
            "plain_ms_per_step": round(ms_plain, 4),
            "batched_over_plain": round(ms_plain / ms, 3),
        },
        "roofline": roof,
        "e2e": {
            "value": round(world * 1000.0 / ms_e2e, 4),
            "unit": "iter/s",
            "h2d_bytes_per_step": int(b.numel() * 4),
            "d2h_bytes_per_step": int(x.data.numel() * 4),
            "api": "SIRT_flatpanel.iterate_from_host(b, x): every step b uploaded from pinned host memory and x "
                   "read back to pinned host memory, the transfers on two copy streams overlapped with the "
                   "neighbouring steps' compute",
        },
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary(),
    }
    if not args.no_batch48 and args.workload == "sirt256":
        # the batched uneven-scan workload at its full ranges, a few iterations
        t0 = time.perf_counter()
        wb = WORKLOADS["batch48"]
        rb = batch48_measure(wb, steps=3, warmup=2, local=local, k_plain=2)
        out["components"]["batch48"] = {
            "workload": f"48 scans, edge log-U{wb['edge']}, views U{wb['views']}, detector U{wb['det']}^2, "
                        "circular/helical with per-view jitter; one SIRT iteration of all scans per step",
            "batched_ms_per_step": round(rb["ms"], 3),
            "per_scan_launch_ms_per_step": round(rb["ms_per_scan"], 3),
            "reference_pattern_ms_per_step": round(rb["ms_ref_pattern"], 3),
            "batched_over_per_scan": round(rb["ms_per_scan"] / rb["ms"], 3),
            "batched_over_reference_pattern": round(rb["ms_ref_pattern"] / rb["ms"], 3),
            "batched_fp_ms": round(rb["t_fp_batch"], 3),
            "batched_bp_ms": round(rb["t_bp_batch"], 3),
            "fwd_rays_per_s": round(rb["stats"]["rays"] / (rb["t_fp_batch"] * 1e-3), 1),
            "back_voxel_updates_per_s": round(rb["stats"]["voxel_views"] / (rb["t_bp_batch"] * 1e-3), 1),
            "steps": 3,
            "section_s": round(time.perf_counter() - t0, 1),
        }
        out["gpu_launches_batch48"] = 2 * 3
    if rank == 0:
        out["rel_l2_vs_fp64"] = parity_check(pg, x, meas, sirt, w)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_reference(pg, x_true, w, b.cpu().numpy(), sirt)
    replicas.finish()
    return out if rank == 0 else {}


def parity_check(pg, x, meas, sirt, w: dict, n_views: int = 8) -> dict:
    """Relative L2 error of the timed operators against the FP64 oracle, outside the timed region.

    On n_views evenly spaced views of the timed scan and the current iterate x:
    the forward projection A_s x, and one SIRT update restricted to those views,
    dx = M (.) B_s(b_s - A_s x), with the same preconditioner M on both sides
    (the reference's update, src/aprict/iterators/sirt_vram.py:130-152).
    """
    import torch

    from aprict_b200.cb import flatpanel as fp
    from oracle import oracle

    n = w["n"]
    corner = -np.float32(w["voxwid"]) * np.array((n, n, n), np.float32) / 2
    sel = np.linspace(0, pg.num_projs, n_views, endpoint=False).astype(int) + 7
    sel = sel % pg.num_projs
    pgs = pg.sliced([int(i) for i in sel])
    specs = pgs.to_proj_spec_array()
    x_np = x.as_numpy().copy()
    t0 = time.perf_counter()
    # forward projection
    ps = fp.ProjectionSet(pgs, data=None)
    fp.project(fp.ConfigProject(), x, ps, block=True)
    want_p, _ = oracle.project_siddon(specs, x_np, voxwid=w["voxwid"], corner=corner)
    err_fp = _rel_l2(ps.data.cpu().numpy(), want_p)
    # one SIRT update on the sampled views: residual kernel + backprojection with M
    b_s = meas.data[torch.as_tensor(sel, device=meas.data.device)].contiguous()
    r = fp.ProjectionSet(pgs, data=None)
    fp.project_residual(fp.ConfigProject(multiply_before_adding=-1), x, r, b_s)
    xn = x.zeroed_copy()
    fp.backproject(sirt._config_bp, xn, r, summand_multiplier=sirt.preconditioner, block=True)  # noqa: SLF001
    r_want = b_s.double().cpu().numpy() - want_p
    mult = sirt.preconditioner.as_numpy().astype(np.float64)
    dx_want = oracle.backproject(specs, r_want, (n, n, n), sirt._config_bp.contents, voxwid=w["voxwid"],  # noqa: SLF001
                                 corner=corner, mult=mult)
    err_res = _rel_l2(r.data.cpu().numpy(), r_want)
    err_dx = _rel_l2(xn.as_numpy(), dx_want)
    return {
        "forward_projection": float(f"{err_fp:.3e}"),
        "residual": float(f"{err_res:.3e}"),
        "sirt_update": float(f"{err_dx:.3e}"),
        "gates": {"projection": 1e-5, "reconstruction": 1e-4},
        "sample": f"{n_views} of {pg.num_projs} views at full detector and volume size; the update is "
                  "M (.) B_s(b_s - A_s x) on those views with the iterate x left by the timed steps",
        "oracle": "FP64 restatement (oracle/ab_oracle.c), OpenMP on the host",
        "check_s": round(time.perf_counter() - t0, 1),
    }


def _rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def workload_text(name: str, w: dict, n_views: int) -> str:
    """The workload string both arms print (one text, so both lines name the same configuration)."""
    return (f"{name}: SIRT iteration, {w['n']}^3 x {w['voxwid']} mm volume, {n_views} views x {w['det']}^2 detector, "
            f"SOD {w['R']} SDD {w['R'] + w['LmR']}")


def cpu_reference(pg, x_true: np.ndarray, w: dict, b: np.ndarray, sirt=None) -> dict:
    """Time one SIRT iteration of the reference's own kernels compiled for the CPU, on a view sample."""
    from aprict_b200.cb import flatpanel as fp
    from oracle import oracle

    kind = "reference" if oracle.have_ref() else "port"
    n = w["n"]
    M = pg.num_projs
    specs = pg.to_proj_spec_array()
    corner = -np.float32(w["voxwid"]) * np.array((n, n, n), np.float32) / 2
    threads = os.cpu_count() or 1
    fp_views = max(1, min(M, int(os.environ.get("APRICT_CPU_FP_VIEWS", "12"))))
    bp_views = max(1, min(M, int(os.environ.get("APRICT_CPU_BP_VIEWS", "10"))))
    x0 = x_true.astype(np.float32)
    sel = np.linspace(0, M, fp_views, endpoint=False).astype(int)
    t0 = time.perf_counter()
    if kind == "reference":
        oracle.ref_project_siddon(specs[sel], x0, voxwid=w["voxwid"], corner=corner, mba=-1.0)
    else:
        oracle.project_siddon(specs[sel], x0, voxwid=w["voxwid"], corner=corner, mba=-1.0)
    t_fp_s = time.perf_counter() - t0
    t_fp = t_fp_s * M / fp_views
    cfg = fp.ConfigBackproject(
        fast_approx=True, cyl_mask_rad=n / 2 * w["voxwid"], apply_summand_multiplier=True, soften_det_edges_proportion=0.05
    )
    mult = np.ones((n, n, n), np.float32)
    vol = np.zeros((n, n, n), np.float32)
    selb = bp_sample_views(M)
    t0 = time.perf_counter()
    if kind == "reference":
        oracle.ref_backproject(specs[selb], b[selb], vol, cfg.contents, voxwid=w["voxwid"], corner=corner, mult=mult)
    else:
        oracle.backproject(specs[selb], b[selb], (n, n, n), cfg.contents, voxwid=w["voxwid"], corner=corner, mult=mult)
    t_bp_s = time.perf_counter() - t0
    t_bp = t_bp_s * M / bp_views
    t_iter = t_fp + t_bp
    return {
        "value": round(1.0 / t_iter, 6),
        "unit": "iter/s",
        "cores": threads,
        "kind": kind,
        "sample": f"projection of {fp_views}/{M} views and backprojection of {bp_views}/{M} views, scaled to the full iteration ({t_fp:.1f} s + {t_bp:.1f} s per iteration)",
        "sampled_views": {"projection": fp_views, "backprojection": bp_views, "of": M},
        "sampled_s": round(t_fp_s + t_bp_s, 3),
        "scale": {"projection": round(M / fp_views, 3), "backprojection": round(M / bp_views, 3)},
    }


def bp_sample_views(M: int) -> np.ndarray:
    """The views the CPU baseline backprojects (evenly spaced)."""
    bp_views = max(1, min(M, int(os.environ.get("APRICT_CPU_BP_VIEWS", "10"))))
    return np.linspace(0, M, bp_views, endpoint=False).astype(int)


def simulate_data_cpu(pg, x_true: np.ndarray, w: dict, views: np.ndarray) -> np.ndarray:
    """The measurement b of the GPU arm's recipe on the given views, computed on the host.

    b = -log(Poisson(I0 exp(-A x_true))/I0), capped at log I0, with A the
    reference's own projector compiled for the CPU; the other views stay zero
    (the CPU sample never reads them). Same phantom, geometry and photon count
    as the GPU arm; the Poisson draws come from numpy's generator with the
    workload's seed.
    """
    from oracle import oracle

    n = w["n"]
    M = pg.num_projs
    corner = -np.float32(w["voxwid"]) * np.array((n, n, n), np.float32) / 2
    specs = pg.to_proj_spec_array()[views]
    if oracle.have_ref():
        p = oracle.ref_project_siddon(specs, x_true, voxwid=w["voxwid"], corner=corner).astype(np.float64)
    else:
        p = oracle.project_siddon(specs, x_true, voxwid=w["voxwid"], corner=corner)[0]
    rng = np.random.default_rng(w["seed"])
    counts = np.maximum(rng.poisson(w["photons"] * np.exp(-p)), 1.0)
    b = np.zeros((M, w["det"], w["det"]), np.float32)
    b[views] = np.minimum(-np.log(counts / w["photons"]), np.log(w["photons"])).astype(np.float32)
    return b


def reference_gpu_sirt(w: dict, steps: int, warmup: int) -> dict:
    """The reference's own GPU kernels on this GPU, in its SIRT iteration's launch pattern.

    The reference's projector and backprojector kernel files, compiled unchanged
    for sm_100a (oracle/_ref/libaprict_refgpu.so), launched as its flatpanel.project
    / flatpanel.backproject launch them (32 x 20 threads per block over the
    detector; 8 x 8 x 8 over the volume, one launch per 10 views), on volumes in
    CUDA arrays behind surfaces. One step is the reference's SIRT iteration
    (src/aprict/iterators/sirt_vram.py:130-152): copy b to the residual, project
    the volume into it with multiply_before_adding = -1 and block, backproject
    it into the volume with the preconditioner and block. The data are the same
    phantom's projection by the reference's own projector with Poisson noise
    (torch's generator, the workload's seed). Nothing of this library runs here.
    """
    import torch

    from oracle import oracle

    torch.cuda.set_device(0)
    n, M = w["n"], w["views"]
    pg, x_true = make_problem(w)
    specs = pg.to_proj_spec_array()
    specs_dev = torch.from_numpy(np.ascontiguousarray(specs).view(np.uint8).copy()).cuda()
    corner = -np.float32(w["voxwid"]) * np.array((n, n, n), np.float32) / 2
    det = w["det"]
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    vw = w["voxwid"]
    # data: the reference's projection of the phantom, Poisson noise at the workload's photon count
    xt = oracle.RefGpuVolume(torch.from_numpy(x_true).cuda().contiguous())
    p = torch.zeros((M, det, det), dtype=torch.float32, device="cuda")
    oracle.ref_gpu_project(xt, specs_dev.data_ptr(), M, det, det, p, voxwid=vw, corner=corner, stream=sp)
    g = torch.Generator(device="cuda").manual_seed(w["seed"])
    counts = torch.poisson(w["photons"] * torch.exp(-p.double()), generator=g).clamp_(min=1.0)
    b = (-torch.log(counts / w["photons"])).clamp_(max=float(np.log(w["photons"]))).float().contiguous()
    del counts, p
    xt.close()
    x = oracle.RefGpuVolume(torch.zeros((n, n, n), dtype=torch.float32, device="cuda"))
    mult = oracle.RefGpuVolume(torch.full((n, n, n), 1e-3, dtype=torch.float32, device="cuda"))
    r = torch.empty_like(b)
    # the reference's config_CB_backproject fields for ConfigBackproject(fast_approx=True,
    # cyl_mask_rad=n/2 voxwid, apply_summand_multiplier=True, soften_det_edges_proportion=0.05)
    cfg = {"exact": 0, "backproject_all_1s": 0, "mask_to_cylinder": 1, "mask_to_cyl_rad": n / 2 * vw,
           "soften_edge_proportion": 0.05, "Z_on_L_factor_power": 0, "Z_on_val_factor_power": 0,
           "Z_on_val_factor_val": 1.0, "approx_mode_direct_raycast": 0, "approx_mode_linear_interpolate": 0,
           "ssx": 1, "ssy": 1, "ssz": 1, "weighting_preset": 0}

    def fp_only() -> None:
        oracle.ref_gpu_project(x, specs_dev.data_ptr(), M, det, det, r, voxwid=vw, corner=corner, mba=-1.0, stream=sp)

    def bp_only() -> None:
        oracle.ref_gpu_backproject(x, specs, r, cfg, voxwid=vw, corner=corner, mult=mult, stream=sp)

    def iterate() -> None:
        r.copy_(b)
        fp_only()
        torch.cuda.synchronize()
        bp_only()
        torch.cuda.synchronize()

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn, k: int) -> float:
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    t_fp = timed(fp_only, 3)
    t_bp = timed(bp_only, 3)
    for _ in range(warmup):
        iterate()
    ms = timed(iterate, steps)
    x.close()
    mult.close()
    rays, vv = M * det * det, n**3 * M
    return {
        "what": "the reference's own GPU kernels (its CB_project_texture_chunked.cu and CB_backproject.cu compiled "
                "unchanged for sm_100a) in its SIRT iteration's launch pattern: copy, projection, 36 ten-view "
                "backprojection launches, two host syncs per iteration",
        "iter_per_s": round(1000.0 / ms, 4),
        "ms_per_step": round(ms, 3),
        "steps": steps,
        "fp_ms": round(t_fp, 3),
        "bp_ms": round(t_bp, 3),
        "fwd_rays_per_s": round(rays / (t_fp * 1e-3), 1),
        "back_voxel_updates_per_s": round(vv / (t_bp * 1e-3), 1),
    }


def run_reference(args) -> dict:
    rank, world, _ = _env_rank()
    if rank != 0:
        return {}
    if args.workload not in ("sirt256", "small"):
        return {"impl": "reference", "unavailable": "the CPU reference arm is timed on the sirt256 workload only"}
    w = WORKLOADS[args.workload]
    pg, x_true = make_problem(w)
    from oracle import oracle

    M = pg.num_projs
    b = simulate_data_cpu(pg, x_true, w, bp_sample_views(M))
    vals = []
    wall = []
    for _ in range(args.warmup):
        cpu_reference(pg, x_true, w, b)
    for _ in range(args.steps):
        t0 = time.perf_counter()
        vals.append(cpu_reference(pg, x_true, w, b))
        wall.append(time.perf_counter() - t0)
    v = statistics.median(c["value"] for c in vals)
    base = dict(vals[0])
    base["value"] = v
    sampled_ms = statistics.median(c["sampled_s"] for c in vals) * 1000.0
    ref_gpu = None
    if not args.no_reference_gpu:
        try:
            import torch

            if torch.cuda.is_available() and oracle.have_ref_gpu():
                ref_gpu = reference_gpu_sirt(w, steps=max(3, min(args.steps, 10)), warmup=2)
            else:
                ref_gpu = {"unavailable": "no GPU or the reference's GPU kernels are not built (oracle/Makefile ref)"}
        except (RuntimeError, OSError) as exc:
            ref_gpu = {"unavailable": f"{type(exc).__name__}: {exc}"[:200]}
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "iter/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1000.0 / v, 3),
        "timing": {
            "kind": "extrapolated",
            "what": "each step times the reference's projector on a view sample and its backprojector on another "
                    "view sample of the full-size iteration; ms_per_step is the time of one whole iteration "
                    "extrapolated from those samples (per-view cost x views), not a timed whole iteration",
            "sampled_ms_per_step": round(sampled_ms, 1),
            "wall_ms_per_step": round(statistics.median(wall) * 1000.0, 1),
            "sampled_views": base["sampled_views"],
            "scale": base["scale"],
        },
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded ellipsoid phantom, simulated Poisson data on the sampled views)",
        "config": {
            "workload": workload_text(args.workload, w, M),
            "baseline_metric": HEADLINE_METRIC,
            "where": "reference device code compiled for the host CPU (oracle/_ref), OpenMP over rays/voxels",
            "oracle_kind": "reference" if oracle.have_ref() else "port",
        },
        "cpu_baseline": base,
        "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": ref_gpu,
    }


def batch48_measure(w: dict, steps: int, warmup: int, local: int, k_plain: int | None = None) -> dict:
    """SIRT over the 48 uneven scans of workload w: batched (graph-replayed
    SIRTBatch) against per-scan launches of the same kernels and against the
    reference's launch pattern. Returns the timings (ms per iteration of all
    scans), the batched component kernels and the workload's sizes."""
    import torch

    from aprict_b200 import Volume, geometry, phantoms
    from aprict_b200.batch import ScanBatch
    from aprict_b200.cb import flatpanel as fp
    from aprict_b200.iterators import SIRT_flatpanel, SIRTBatch

    rng = np.random.default_rng(w["seed"])
    params = geometry.uneven_scans(rng, w["n_scans"], edge=w["edge"], views=w["views"], det=w["det"],
                                   voxwid=w["voxwid"], R=w["R"], L_minus_R=w["LmR"])
    sirts, truths = [], []
    stats = dict(rays=0, voxel_views=0, voxels=0, proj_bytes=0)
    for i, sp in enumerate(params):
        n = sp["n"]
        pg = geometry.scan_geometry(rng, sp)
        xt = phantoms.ellipsoid_volume(w["seed"] * 1000 + i, w["n_ellipsoids"], (n, n, n), w["voxwid"],
                                       semi_axes_vox=(max(2.0, n / 32), n / 6))
        v = Volume(xt, voxwid=w["voxwid"])
        ps = fp.ProjectionSet(pg, data=None)
        fp.project(fp.ConfigProject(), v, ps)
        g = torch.Generator(device="cuda").manual_seed(w["seed"] + i)
        lam = w["photons"] * torch.exp(-ps.data.double())
        counts = torch.poisson(lam, generator=g).clamp_(min=1.0)
        b = (-torch.log(counts / w["photons"])).clamp_(max=float(np.log(w["photons"]))).float()
        del lam, counts, v
        sirts.append(SIRT_flatpanel(SIRT_flatpanel.Config(), Volume.zeros((n, n, n), voxwid=w["voxwid"]),
                                    fp.ProjectionSet(pg, data=b)))
        stats["rays"] += sp["views"] * sp["det"] ** 2
        stats["voxel_views"] += n**3 * sp["views"]
        stats["voxels"] += n**3
        stats["proj_bytes"] += 4 * sp["views"] * sp["det"] ** 2
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn, k: int) -> float:
        torch.cuda.synchronize()
        s, e = ev(), ev()
        s.record(stream)
        for _ in range(k):
            fn()
        e.record(stream)
        torch.cuda.synchronize()
        return s.elapsed_time(e) / k

    # components: one batched projection (residual) and one batched backprojection
    vols = [s.volume for s in sirts]
    rs = [s._scratch for s in sirts]  # noqa: SLF001
    batch = ScanBatch(vols, rs)
    fp_plan = batch.plan_project(fp.ConfigProject(multiply_before_adding=-1), bases=[s._meas.data for s in sirts])  # noqa: SLF001
    bp_plan = batch.plan_backproject([s._config_bp for s in sirts], multipliers=[s.preconditioner for s in sirts])  # noqa: SLF001
    fp_plan.run()
    bp_plan.run()
    t_fp_batch = timed(fp_plan.run, 2)
    t_bp_batch = timed(bp_plan.run, 2)

    # batched SIRT (graph replay), the headline
    sb = SIRTBatch(sirts)
    sb.iterate_graph(1)
    for _ in range(max(0, warmup - 1)):
        sb.iterate_graph(1)
    with ClockSampler(local) as clk:
        ms = timed(lambda: sb.iterate_graph(1), steps)

    # per-scan launches of the same kernels (no host synchronisation)
    cfg_res = fp.ConfigProject(multiply_before_adding=-1)

    def per_scan_iter() -> None:
        for s in sirts:
            s.iterate()

    per_scan_iter()
    k_plain = k_plain or max(2, steps // 2)
    ms_per_scan = timed(per_scan_iter, k_plain)

    # the reference's launch pattern per scan
    chunks = []
    for s in sirts:
        pg = s._meas.proj_geom  # noqa: SLF001
        r = s._scratch  # noqa: SLF001
        chunks.append([fp.ProjectionSet(pg.sliced(slice(c0, min(c0 + 10, pg.num_projs))),
                                        data=r.data[c0:min(c0 + 10, pg.num_projs)])
                       for c0 in range(0, pg.num_projs, 10)])
    cfg_acc = fp.ConfigProject(multiply_before_adding=-1)

    def ref_pattern_iter() -> None:
        for s, ch in zip(sirts, chunks):
            s._scratch.data.copy_(s._meas.data)  # noqa: SLF001
            fp.project(cfg_acc, s.volume, s._scratch, block=True)  # noqa: SLF001
            for c in ch:
                fp.backproject(s._config_bp, s.volume, c, summand_multiplier=s.preconditioner)  # noqa: SLF001
            torch.cuda.synchronize()

    ref_pattern_iter()
    ms_ref_pattern = timed(ref_pattern_iter, k_plain)
    del cfg_res

    return dict(ms=ms, ms_per_scan=ms_per_scan, ms_ref_pattern=ms_ref_pattern, t_fp_batch=t_fp_batch,
                t_bp_batch=t_bp_batch, stats=stats, n_scans=len(sirts), clocks=clk.summary())


def run_batch(args) -> dict:
    """Workload batch48: SIRT over 48 uneven scans, batched vs plain launches.

    A step is one SIRT iteration of all 48 scans. ``value`` is the batched
    form (SIRTBatch: two persistent launches per iteration, replayed from a
    CUDA graph). Beside it: the same kernels launched per scan (fused residual
    + all-view backprojection, 96 launches per iteration) and the reference's
    launch pattern per scan (copy, accumulate projection, 10-view
    backprojection launches, a host synchronisation per scan).
    """
    import torch

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    r = batch48_measure(w, args.steps, args.warmup, local)
    ms, ms_per_scan, ms_ref_pattern = r["ms"], r["ms_per_scan"], r["ms_ref_pattern"]
    t_fp_batch, t_bp_batch, stats, n_scans = r["t_fp_batch"], r["t_bp_batch"], r["stats"], r["n_scans"]
    peak, peak_kind = load_peaks()
    out = {
        "metric": "batched SIRT iter/s (48 uneven scans per iteration)",
        "value": round(1000.0 / ms, 4),
        "unit": "iter/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded ellipsoid phantoms, simulated Poisson data)",
        "config": {
            "workload": f"batch48: SIRT iteration over {n_scans} scans, edge log-U{w['edge']}, views U{w['views']}, "
                        f"detector U{w['det']}^2, circular/helical with per-view jitter",
            "baseline_metric": HEADLINE_METRIC,
            "parallelism": "1 GPU",
            "l2": f"inputs larger than L2 (projections {stats['proj_bytes'] / 1e9:.1f} GB x2)",
            "form": "batched: SIRTBatch, two persistent launches per iteration, CUDA-graph replay",
        },
        "components": {
            "batched_fp_ms": round(t_fp_batch, 3),
            "batched_bp_ms": round(t_bp_batch, 3),
            "fwd_rays_per_s": round(stats["rays"] / (t_fp_batch * 1e-3), 1),
            "back_voxel_updates_per_s": round(stats["voxel_views"] / (t_bp_batch * 1e-3), 1),
            "per_scan_launch_ms_per_step": round(ms_per_scan, 3),
            "reference_pattern_ms_per_step": round(ms_ref_pattern, 3),
            "batched_over_per_scan": round(ms_per_scan / ms, 3),
            "batched_over_reference_pattern": round(ms_ref_pattern / ms, 3),
            "workload_fp_bp_20iter_s": round((t_fp_batch + t_bp_batch + 20 * ms) / 1000.0, 3),
            "rays": stats["rays"],
            "voxel_views": stats["voxel_views"],
        },
        "roofline": {
            "bound": "hbm",
            "kernel": "batched backproject",
            "achieved": round((4.0 * stats["voxel_views"] + 12.0 * stats["voxels"]) / (t_bp_batch * 1e-3) / 1e9, 1),
            "peak": peak,
            "unit": "GB/s",
            "frac": round((4.0 * stats["voxel_views"] + 12.0 * stats["voxels"]) / (t_bp_batch * 1e-3) / 1e9 / peak, 4),
            "traffic": None,
            "peak_kind": peak_kind,
        },
        "e2e": None,
        "gpu_launches": 2 * args.steps,
        "clocks": r["clocks"],
    }
    return out if rank == 0 else {}


def _timed(fn, k: int) -> float:
    import torch

    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(k):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / k


def _line(args, metric: str, value: float, unit: str, ms: float, workload: str, extra: dict) -> dict:
    out = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded phantoms)", "config": {"workload": workload, "baseline_metric": HEADLINE_METRIC},
    }
    out.update(extra)
    return out


def quadric_tests(pg, shapes: np.ndarray, tile: int = 16) -> tuple[int, int]:
    """Ray-shape tests of the analytic projector after its tile cull, and their FP64 FLOPs.

    The cull restated on the host: per view, each shape's world bounding box
    (8 corners, from the compiled quadrics) is projected onto the detector and
    kept for every 16 x 16 pixel tile its footprint meets (the whole detector
    when a corner is not in front of the source); every ray of a kept tile
    tests the shape. FLOPs per test are the kernel's FP64 operations on the hit
    path (a division or square root counting one): 12 for the ray direction in
    the shape's frame, 17 (ellipsoid) or 18 (cylinder) for the quadric roots, 5
    per clip plane and 3 for the additive accumulation.
    """
    from aprict_b200.cb import forbild

    q = forbild.compile_shapes(shapes)
    kind, nclip = q["kind"], q["n_clip"] & 0xFF
    c = np.array([list(x) for x in q["c"]], np.float64)
    bb = np.array([list(x) for x in q["bb_half"]], np.float64)
    sgn = np.array([[(1 if k & 4 else -1), (1 if k & 2 else -1), (1 if k & 1 else -1)] for k in range(8)], np.float64)
    X = c[:, None, :] + sgn[None] * bb[:, None, :]
    flops_pair = np.where(kind == 1, 12 + 17, 12 + 18) + 5 * nclip + 3
    flops_pair = np.where(kind == 0, 0, flops_pair)
    specs = pg.to_proj_spec_array()
    pairs = flops = 0
    for sp in specs:
        s = np.array([sp["source_pos"][k] for k in "xyz"], np.float64)
        P = np.array([sp["det_pos"][k] for k in "xyz"], np.float64)  # noqa: N806
        U = np.array([sp["det_u"][k] for k in "xyz"], np.float64)  # noqa: N806
        V = np.array([sp["det_v"][k] for k in "xyz"], np.float64)  # noqa: N806
        nu, nv = int(sp["nu"]), int(sp["nv"])
        n = np.cross(U, V)
        Ps = P - s  # noqa: N806
        Dn = Ps @ n  # noqa: N806
        Au = (U * Dn - n * (U @ Ps)) / (U @ U) + n * (nu - 1) / 2  # noqa: N806
        Av = (V * Dn - n * (V @ Ps)) / (V @ V) + n * (nv - 1) / 2  # noqa: N806
        r = X - s
        den = r @ n
        fu, fv = (r @ Au) / den, (r @ Av) / den
        front = np.all(den * np.sign(Dn) > 0, axis=1)
        tu = np.arange((nu + tile - 1) // tile)
        tv = np.arange((nv + tile - 1) // tile)
        u0, u1 = tu * tile - 0.5, np.minimum(nu, (tu + 1) * tile) - 0.5
        v0, v1 = tv * tile - 0.5, np.minimum(nv, (tv + 1) * tile) - 0.5
        ku = (fu.max(1)[:, None] >= u0[None] - 1e-6) & (fu.min(1)[:, None] <= u1[None] + 1e-6) | ~front[:, None]
        kv = (fv.max(1)[:, None] >= v0[None] - 1e-6) & (fv.min(1)[:, None] <= v1[None] + 1e-6) | ~front[:, None]
        rays_u = (np.minimum(nu, (tu + 1) * tile) - tu * tile)[None, :]
        rays_v = (np.minimum(nv, (tv + 1) * tile) - tv * tile)[None, :]
        tests = (ku * rays_u).sum(1) * (kv * rays_v).sum(1) * (kind != 0)
        pairs += int(tests.sum())
        flops += int((tests * flops_pair).sum())
    return pairs, flops


def run_component(args) -> dict:
    """The fpbp128, fbp64 and quadric workloads (component measurements)."""
    import torch

    from aprict_b200 import FBVolume, Volume, phantoms
    from aprict_b200.cb import flatpanel as fp
    from aprict_b200.recon import fbp_fan_circ, fbp_fan_circ_batch

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    peak, peak_kind = load_peaks()
    if args.workload == "fpbp128":
        n = w["n"]
        pg = fp.ProjGeom.new_circular_scan(num_source_points=w["views"], R=w["R"], L_minus_R=w["LmR"],
                                           pix_widhei_at_isocenter=(w["pix_at_iso"],) * 2, num_pix_widhei=(w["det"],) * 2)
        x = Volume(phantoms.ellipsoid_volume(w["seed"], w["n_ellipsoids"], (n, n, n), w["voxwid"], semi_axes_vox=(5, 40)),
                   voxwid=w["voxwid"])
        ps = fp.ProjectionSet(pg, data=None)
        ps.create_buffer()
        y = fp.ProjectionSet(pg, data=torch.rand_like(ps.data))
        rays, vv = w["views"] * w["det"] ** 2, n**3 * w["views"]
        t_fp = _timed(lambda: fp.project(fp.ConfigProject(), x, ps), args.steps)
        out_v = Volume.zeros((n, n, n), voxwid=w["voxwid"])
        t_ex = _timed(lambda: fp.backproject(fp.ConfigBackproject(), out_v, y), args.steps)
        t_near = _timed(lambda: fp.backproject(fp.ConfigBackproject(fast_approx=True), out_v, y), args.steps)
        t_lin = _timed(lambda: fp.backproject(fp.ConfigBackproject(fast_approx=True, approx_mode_bilinear_interpolate=True),
                                              out_v, y), args.steps)
        t_adj = _timed(lambda: fp.backproject_adjoint(fp.ConfigProject(), out_v, y), args.steps)
        nseg, _ = count_segments(pg, (n, n, n), w["voxwid"])
        fp_gbs = (4.0 * nseg + 4.0 * rays) / (t_fp * 1e-3) / 1e9
        extra = {
            "components": {
                "fp_ms": round(t_fp, 4), "bp_exact_ms": round(t_ex, 4), "bp_fast_nearest_ms": round(t_near, 4),
                "bp_fast_bilinear_ms": round(t_lin, 4), "adjoint_scatter_ms": round(t_adj, 4),
                "fwd_rays_per_s": round(rays / (t_fp * 1e-3), 1),
                "back_exact_voxel_updates_per_s": round(vv / (t_ex * 1e-3), 1),
                "back_fast_voxel_updates_per_s": round(vv / (t_near * 1e-3), 1),
            },
            "roofline": {"bound": "hbm", "kernel": "project_siddon", "achieved": round(fp_gbs, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(fp_gbs / peak, 4), "traffic": None, "peak_kind": peak_kind},
        }
        if not args.no_cpu_baseline:
            from oracle import oracle

            sel = np.linspace(0, w["views"], 6, endpoint=False).astype(int)
            corner = -np.float32(w["voxwid"]) * np.array((n, n, n), np.float32) / 2
            t0 = time.perf_counter()
            (oracle.ref_project_siddon if oracle.have_ref() else oracle.project_siddon)(
                pg.to_proj_spec_array()[sel], x.as_numpy(), voxwid=w["voxwid"], corner=corner)
            dt = time.perf_counter() - t0
            extra["cpu_baseline"] = {"value": round(len(sel) * w["det"] ** 2 / dt, 1), "unit": "rays/s",
                                     "cores": os.cpu_count() or 1, "kind": "reference" if oracle.have_ref() else "port",
                                     "sample": f"forward projection of {len(sel)} of {w['views']} views"}
        return _line(args, "fwd rays/s", round(rays / (t_fp * 1e-3), 1), "rays/s", t_fp,
                     f"fpbp128: {n}^3 x {w['voxwid']} mm, {w['views']} views x {w['det']}^2", extra)
    if args.workload == "fbp64":
        n, S, m, nu = w["n"], w["slices"], w["views"], w["det"]
        L = w["R"] + w["LmR"]  # noqa: N806
        pg = fp.ProjGeom.new_circular_scan(num_source_points=m, R=w["R"], L_minus_R=w["LmR"],
                                           pix_widhei_at_isocenter=(w["pix"] * w["R"] / L,) * 2, num_pix_widhei=(nu, 1))
        projs = []
        for k in range(S):
            xs = phantoms.ellipsoid_volume(w["seed"] * 100 + k, w["n_ellipses"], (n, n, 1), w["voxwid"],
                                           semi_axes_vox=(8, 160), rho=(0.05, 1.0))
            ps = fp.ProjectionSet(pg, data=None)
            fp.project(fp.ConfigProject(), Volume(xs, voxwid=w["voxwid"]), ps)
            projs.append(ps)
        stacked = torch.cat([p.data for p in projs], dim=0)
        vols = [Volume.zeros((n, n, 1), voxwid=w["voxwid"]) for _ in range(S)]
        t_b = _timed(lambda: fbp_fan_circ_batch(projs, vols, apodization="hann", stacked=stacked), args.steps)

        def per_slice() -> None:
            for p, v in zip(projs, vols):
                fbp_fan_circ(p, v, apodization="hann")

        t_s = _timed(per_slice, max(1, args.steps // 2))
        vv = S * n * n * m
        extra = {"components": {"batched_ms": round(t_b, 3), "per_slice_ms": round(t_s, 3),
                                "batched_over_per_slice": round(t_s / t_b, 3),
                                "back_voxel_updates_per_s": round(vv / (t_b * 1e-3), 1),
                                "filtered_samples_per_s": round(S * m * nu / (t_b * 1e-3), 1)}}
        return _line(args, "fan FBP slices/s", round(S / (t_b * 1e-3), 2), "slices/s", t_b,
                     f"fbp64: {S} slices {n}^2 x {w['voxwid']} mm, {m} views x {nu} x {w['pix']} mm, Ram-Lak + Hann", extra)
    if args.workload in ("fbpcyl", "gbc"):
        return _run_cylinder_recon(args, w)
    # quadric
    shapes = phantoms.random_quadric_phantom(w["seed"], n_ellipsoids=w["n_ellipsoids"], n_cylinders=w["n_cylinders"],
                                             radius=w["radius"])
    L = w["R"] + w["LmR"]  # noqa: N806
    pg = fp.ProjGeom.new_circular_scan(num_source_points=w["views"], R=w["R"], L_minus_R=w["LmR"],
                                       pix_widhei_at_isocenter=(w["pix"] * w["R"] / L,) * 2, num_pix_widhei=(w["det"],) * 2)
    ps = fp.ProjectionSet(pg, data=None)
    ps.create_buffer()
    vol = FBVolume(shapes)
    cfg = fp.ConfigProject(overlap_addition=True)
    t_q = _timed(lambda: fp.project(cfg, vol, ps), args.steps)
    rays = w["views"] * w["det"] ** 2
    pairs, flops = quadric_tests(pg, shapes)
    fp64_peak = 148 * 64 * 2 * 1.965e9  # nominal FP64 FLOP/s (SMs x FP64 lanes x 2 x max SM clock)
    extra = {"components": {"project_ms": round(t_q, 3), "rays_per_s": round(rays / (t_q * 1e-3), 1),
                            "overflow_rays": int(ps.out_of_mem_count),
                            "output_GB": round(4 * rays / 1e9, 3),
                            "output_write_GBps": round(4 * rays / (t_q * 1e-3) / 1e9, 1),
                            "ray_shape_tests": pairs,
                            "fp64_flops_algorithmic": flops,
                            "fp64_tflops_algorithmic": round(flops / (t_q * 1e-3) / 1e12, 3),
                            "fp64_frac_of_nominal_peak": round(flops / (t_q * 1e-3) / fp64_peak, 4)}}
    return _line(args, "quadric projection rays/s", round(rays / (t_q * 1e-3), 1), "rays/s", t_q,
                 f"quadric: {len(shapes)} clipped quadrics in {2 * w['radius']:.0f} mm, {w['views']} views x {w['det']}^2 x {w['pix']} mm, additive", extra)


def _run_cylinder_recon(args, w: dict) -> dict:
    """The fbpcyl and gbc workloads: one full reconstruction per step, with its parts timed apart."""
    import torch  # noqa: F401

    from aprict_b200 import Volume, geometry, phantoms
    from aprict_b200.cb import flatpanel as fp
    from aprict_b200.cb.ramp_filter import FBPFilterer
    from aprict_b200.gbc import weightinteg
    from aprict_b200.recon import fan_geometry, fbp_cone_cyl, gbc_cone_cyl

    n, vw, m = w["n"], w["voxwid"], w["views"]
    pg = geometry.cylinder_scan(n_views=m, R=w["R"], L_minus_R=w["LmR"], pix_at_iso=w["pix_at_iso"], nu=w["det"],
                                nv=w["det"], height=w["height"])
    x = Volume(phantoms.ellipsoid_volume(w["seed"], w["n_ellipsoids"], (n, n, n), vw, semi_axes_vox=(3, n / 5)),
               voxwid=vw)
    ps = fp.ProjectionSet(pg, data=None)
    fp.project(fp.ConfigProject(), x, ps, block=True)
    R, L, pixwid, nu, nv = fan_geometry(pg)  # noqa: N806
    steps = max(1, args.steps)

    if args.workload == "fbpcyl":
        out = Volume.zeros((n, n, n), voxwid=vw)
        t_all = _timed(lambda: fbp_cone_cyl(ps, out, seed_proj_rots=1, num_projs_per_chunk=m), steps)
        filt = FBPFilterer(L=L, physpixwid=pixwid, proj_2d_shape=(nu, nv), projs_per_batch=m,
                           rng=np.random.default_rng(1))
        t_f = _timed(lambda: filt.filter_bulk_axis1_concat(ps.data, block=False), steps)
        (filtered,), _ = filt.filter_bulk_axis1_concat(ps.data)
        support = R * np.sin(np.arctan(pixwid * nu / 2 / L))
        cfg = fp.ConfigBackproject(fast_approx=True, cyl_mask_rad=support, Z_on_val_factor_power=-3,
                                   Z_on_val_factor_val=R, approx_mode_direct_raycast=True)
        fps = fp.ProjectionSet(pg, data=filtered)
        t_bp = _timed(lambda: fp.backproject(cfg, out, fps), steps)
        vv = n**3 * m
        extra = {"components": {"recon_ms": round(t_all, 3), "tilted_filter_ms": round(t_f, 3),
                                "backproject_ms": round(t_bp, 3),
                                "back_voxel_updates_per_s": round(vv / (t_bp * 1e-3), 1),
                                "filtered_views_per_s": round(m / (t_f * 1e-3), 1)}}
        from oracle import oracle  # the CPU baseline leg

        if not args.no_cpu_baseline and oracle.have_ref():
            sel = np.linspace(0, m, 4, endpoint=False).astype(int)
            corner = -np.float32(vw) * np.array((n, n, n), np.float32) / 2
            v = np.zeros((n, n, n), np.float32)
            f_host = filtered.cpu().numpy()[sel]
            t0 = time.perf_counter()
            oracle.ref_backproject(pg.to_proj_spec_array()[sel], f_host, v, cfg.contents, voxwid=vw, corner=corner)
            dt = time.perf_counter() - t0
            extra["cpu_baseline"] = {"value": round(len(sel) * n**3 / dt, 1), "unit": "voxel-updates/s",
                                     "cores": os.cpu_count() or 1, "kind": "reference",
                                     "sample": f"direct-raycast backprojection of {len(sel)} of {m} views "
                                               "(the reference's filter runs on the GPU through cupyx: no CPU arm)"}
        return _line(args, "cone-cylinder FBP reconstructions/s", round(1000.0 / t_all, 3), "recon/s", t_all,
                     f"fbpcyl: {n}^3 x {vw} mm, {m} golden-angle views on R {w['R']} mm x {w['height']} mm, "
                     f"{nu}^2 x {pixwid:.2f} mm, one random filter rotation per view", extra)
    # gbc
    t_all = _timed(lambda: gbc_cone_cyl(ps, (n, n, n), vw), steps)
    vartheta_v = float(np.arctan2(nv * pixwid / 2 - pixwid / 2, np.sqrt(L**2 + (nu * pixwid / 2 - pixwid / 2) ** 2)))
    vartheta_h = float(np.arctan2(nu * pixwid / 2 - pixwid / 2, L))
    cfg = fp.ConfigBackproject(fast_approx=True, Z_on_val_factor_val=R, backproj_weighting_preset=7,
                               approx_mode_direct_raycast=True, approx_mode_bilinear_interpolate=True,
                               soft_vartheta_v=vartheta_v, soft_vartheta_v_softspan=0.05, soft_vartheta_h=vartheta_h,
                               soft_vartheta_h_softspan=0.05)
    pad = 9 * (4 + int(np.ceil(n * 1.2 / 9)))
    pad = pad if (pad - n) % 2 == 0 else pad + 9
    vol, ws = Volume.zeros((pad,) * 3, voxwid=vw), Volume.zeros((pad,) * 3, voxwid=vw)
    t_bp = _timed(lambda: fp.backproject(cfg, vol, ps, secondary_volume=ws), steps)
    xs = vol.xs_ys_zs[0]
    t_wi = _timed(lambda: weightinteg.backproj_gbc_weight_integ_xygrid_GPU(xs, xs, R, cfg), steps)
    vv = pad**3 * m
    extra = {"components": {"recon_ms": round(t_all, 3), "gbc_backproject_padded_ms": round(t_bp, 3),
                            "weight_integral_ms": round(t_wi, 3), "padded_edge": pad,
                            "gbc_voxel_updates_per_s": round(vv / (t_bp * 1e-3), 1)}}
    from oracle import oracle  # the CPU baseline leg

    if not args.no_cpu_baseline and oracle.have_ref():
        sel = np.array([0, m // 2])
        v1, v2 = np.zeros((pad,) * 3, np.float32), np.zeros((pad,) * 3, np.float32)
        t0 = time.perf_counter()
        oracle.ref_backproject_gbc(pg.to_proj_spec_array()[sel], ps.data.cpu().numpy()[sel], v1, v2, cfg.contents,
                                   voxwid=vw, corner=vol.corner)
        dt = time.perf_counter() - t0
        extra["cpu_baseline"] = {"value": round(len(sel) * pad**3 / dt, 1), "unit": "voxel-updates/s",
                                 "cores": os.cpu_count() or 1, "kind": "reference",
                                 "sample": f"GBC backprojection of {len(sel)} of {m} views into the {pad}^3 padded volume"}
    return _line(args, "GBC reconstructions/s", round(1000.0 / t_all, 4), "recon/s", t_all,
                 f"gbc: {n}^3 x {vw} mm, {m} golden-angle views on R {w['R']} mm x {w['height']} mm, "
                 f"{nu}^2 x {pixwid:.2f} mm, n 9, f1 1.2, f2 6", extra)


def profile_kernels(args) -> dict:
    """Launch the workload's kernels a few times and exit (a small driver for ncu captures).

    Launch order: 1 projection (simulated data), then ``--steps`` x (fused
    residual projection, all-view backprojection); nothing else runs on the GPU.
    quadric, fbp64, fbpcyl and gbc launch their own workload's kernels instead.
    """
    import torch

    from aprict_b200 import FBVolume, Volume, phantoms
    from aprict_b200.cb import flatpanel as fp

    w = WORKLOADS[args.workload]
    if args.workload == "quadric":  # 4 views of the quadric workload: one analytic-projector launch per step
        L = w["R"] + w["LmR"]  # noqa: N806
        pg = fp.ProjGeom.new_circular_scan(num_source_points=4, R=w["R"], L_minus_R=w["LmR"],
                                           pix_widhei_at_isocenter=(w["pix"] * w["R"] / L,) * 2,
                                           num_pix_widhei=(w["det"],) * 2)
        ps = fp.ProjectionSet(pg, data=None)
        vol = FBVolume(phantoms.random_quadric_phantom(w["seed"], n_ellipsoids=w["n_ellipsoids"],
                                                       n_cylinders=w["n_cylinders"], radius=w["radius"]))
        for _ in range(args.steps):
            fp.project(fp.ConfigProject(overlap_addition=True), vol, ps)
        torch.cuda.synchronize()
        return {"mode": "kernels", "workload": args.workload, "launches": args.steps}
    if args.workload == "fbp64":  # 8 slices: one ramp-filter launch and one batched backprojection per step
        from aprict_b200.recon import fbp_fan_circ_batch

        L = w["R"] + w["LmR"]  # noqa: N806
        pg = fp.ProjGeom.new_circular_scan(num_source_points=w["views"], R=w["R"], L_minus_R=w["LmR"],
                                           pix_widhei_at_isocenter=(w["pix"] * w["R"] / L,) * 2,
                                           num_pix_widhei=(w["det"], 1))
        projs = [fp.ProjectionSet(pg, data=torch.rand((w["views"], w["det"], 1), device="cuda")) for _ in range(8)]
        vols = [Volume.zeros((w["n"], w["n"], 1), voxwid=w["voxwid"]) for _ in range(8)]
        for _ in range(args.steps):
            fbp_fan_circ_batch(projs, vols, apodization="hann")
        torch.cuda.synchronize()
        return {"mode": "kernels", "workload": args.workload, "launches": 2 * args.steps}
    if args.workload == "gbc":  # per step: one GBC backprojection of the padded volume, one weight integral
        from aprict_b200 import geometry
        from aprict_b200.gbc import weightinteg

        n, m, vw = w["n"], w["views"], w["voxwid"]
        pg = geometry.cylinder_scan(n_views=m, R=w["R"], L_minus_R=w["LmR"], pix_at_iso=w["pix_at_iso"],
                                    nu=w["det"], nv=w["det"], height=w["height"])
        gen = torch.Generator(device="cuda")
        gen.manual_seed(w["seed"])
        ps = fp.ProjectionSet(pg, data=torch.rand((m, w["det"], w["det"]), device="cuda", generator=gen))
        L = w["R"] + w["LmR"]  # noqa: N806
        pixwid = float(np.linalg.norm(pg.det_uvec[0]))
        nu = nv = w["det"]
        cfg = fp.ConfigBackproject(
            fast_approx=True, Z_on_val_factor_val=w["R"], backproj_weighting_preset=7, approx_mode_direct_raycast=True,
            approx_mode_bilinear_interpolate=True,
            soft_vartheta_v=float(np.arctan2(nv * pixwid / 2 - pixwid / 2, np.sqrt(L**2 + (nu * pixwid / 2 - pixwid / 2) ** 2))),
            soft_vartheta_v_softspan=0.05, soft_vartheta_h=float(np.arctan2(nu * pixwid / 2 - pixwid / 2, L)),
            soft_vartheta_h_softspan=0.05)
        pad = 9 * (4 + int(np.ceil(n * 1.2 / 9)))
        pad = pad if (pad - n) % 2 == 0 else pad + 9
        vol, ws = Volume.zeros((pad,) * 3, voxwid=vw), Volume.zeros((pad,) * 3, voxwid=vw)
        xs = vol.xs_ys_zs[0]
        for _ in range(args.steps):
            fp.backproject(cfg, vol, ps, secondary_volume=ws)
            weightinteg.backproj_gbc_weight_integ_xygrid_GPU(xs, xs, w["R"], cfg)
        torch.cuda.synchronize()
        return {"mode": "kernels", "workload": args.workload, "launches": 2 * args.steps}
    if args.workload == "fbpcyl":  # one direct-raycast backprojection of the cone-cylinder FBP per step
        from aprict_b200 import geometry

        n, m = w["n"], w["views"]
        pg = geometry.cylinder_scan(n_views=m, R=w["R"], L_minus_R=w["LmR"], pix_at_iso=w["pix_at_iso"],
                                    nu=w["det"], nv=w["det"], height=w["height"])
        gen = torch.Generator(device="cuda")
        gen.manual_seed(w["seed"])
        ps = fp.ProjectionSet(pg, data=torch.rand((m, w["det"], w["det"]), device="cuda", generator=gen))
        L = w["R"] + w["LmR"]  # noqa: N806
        pixwid = float(np.linalg.norm(pg.det_uvec[0]))
        cfg = fp.ConfigBackproject(fast_approx=True, cyl_mask_rad=w["R"] * np.sin(np.arctan(pixwid * w["det"] / 2 / L)),
                                   Z_on_val_factor_power=-3, Z_on_val_factor_val=w["R"], approx_mode_direct_raycast=True)
        out = Volume.zeros((n, n, n), voxwid=w["voxwid"])
        for _ in range(args.steps):
            fp.backproject(cfg, out, ps)
        torch.cuda.synchronize()
        return {"mode": "kernels", "workload": args.workload, "launches": args.steps}
    n = w["n"]
    pg, x_true = make_problem(w)
    b = simulate_data(pg, x_true, w)
    meas = fp.ProjectionSet(pg, data=b)
    x = Volume(x_true * 0.5, voxwid=w["voxwid"])
    M = Volume(np.full((n, n, n), 1e-3, np.float32), voxwid=w["voxwid"])  # noqa: N806
    r = meas.zeroed_copy()
    cfg_bp = fp.ConfigBackproject(
        fast_approx=True, cyl_mask_rad=n / 2 * w["voxwid"], apply_summand_multiplier=True, soften_det_edges_proportion=0.05
    )
    for _ in range(args.steps):
        fp.project_residual(fp.ConfigProject(multiply_before_adding=-1), x, r, meas.data)
        fp.backproject(cfg_bp, x, r, summand_multiplier=M)
    torch.cuda.synchronize()
    return {"mode": "kernels", "workload": args.workload, "launches": 1 + 2 * args.steps}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="sirt256")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch48", action="store_true", help="skip the batched uneven-scan section of the default line")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own kernels on the GPU")
    ap.add_argument("--mode", choices=["bench", "kernels"], default="bench")
    ap.add_argument("--tuning", default="",
                    help="--mode kernels only: tile-shape knobs for A/B captures, e.g. fp_tile_v=16,fp_warp_v=16 "
                         "(the names of aprict_b200.autotune)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.tuning and args.mode != "kernels":
        ap.error("--tuning applies to --mode kernels only")
    if args.mode == "kernels":
        if args.tuning:
            from aprict_b200 import autotune

            knobs = {k: int(v) for k, v in (kv.split("=") for kv in args.tuning.split(","))}
            known = {"fp_tile_v", "fp_warp_v", "fp_views", "fp_warp_views", "bp_xb", "bp_wave", "fp_ss1", "bp_zlanes"}
            if set(knobs) - known:
                ap.error(f"--tuning: unknown knobs {sorted(set(knobs) - known)}")
            autotune.apply(knobs)
        out = profile_kernels(args)
    else:
        if args.impl == "reference":
            out = run_reference(args)
        elif args.workload == "batch48":
            out = run_batch(args)
        elif args.workload in ("fpbp128", "fbp64", "quadric", "fbpcyl", "gbc"):
            out = run_component(args)
        else:
            out = run_ours(args)
    if out:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
