"""Benchmark of the B200 PatchStereo engine on the drone-scale workload (1920×1080, 24 views).

One step = the whole depth-map schedule of every view of the job: photometric run from random init (6 red-black
iterations), one geometric-consistency round (2 iterations against the snapshot of all views), the geometric filter
and the readout threshold.  `value` = views/s of the whole job with every input resident in HBM; `e2e` = the same
through the reference-facing C ABI with host buffers (session begin = image upload, host states in and out, host
snapshots, host counts) inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--math parity|fast] [--impl ours|reference]

N > 1 (torchrun): by default every rank runs its own 24-view job (a differently seeded scene) with no collective in
the data path ("scaling": "weak"); with --shard-job the views of ONE job are sharded over ranks (by pixel count)
and the geometric round's snapshot is exchanged per owner rank over NCCL into every GPU's own snapshot buffer
("scaling": "strong").  `--impl reference` times the CPU
oracle (this project's C++ restatement of the reference kernel; the reference has no CPU path of its own) on the
host cores, on a bounded sample (one view, one iteration) of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOP_PER_TAP_CACHED = 33  # NCC tap with cached weights: projection 15 + bilinear 12 + accumulation 6 (FMA = 2)


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_workload(args, rank: int, shard_job: bool):
    """The benchmark workload: c2 (drone scale, the metric's configuration; default), c1 (640×480, 3 views) or c3
    (64 views of mixed sizes from 4 terrains, 2-8 sources each)."""
    from cumulus3d_b200 import scenes
    seed_shift = 0 if shard_job else rank
    if args.workload == "c1":
        return scenes.workload_c1(seed=1 + seed_shift)
    if args.workload == "c3":
        return scenes.workload_c3(seed=3 + seed_shift)
    if args.workload == "c5":
        return scenes.workload_c5(seed=5 + seed_shift, views=args.views)
    return scenes.workload_c2(seed=2 + seed_shift, with_gt=False, views=args.views)


def bench_config(wl, world: int, shard_job: bool, math: str) -> dict:
    """The `config` of the line, the same in both arms (the reference arm times this workload on the CPU oracle)."""
    wn = 2 * wl.input.pm.window_radius // wl.input.pm.window_step + 1
    views_total = len(wl.cams) * (1 if shard_job else world)
    return {"workload": wl.name, "views": views_total, "sizes": sorted({f"{c.width}x{c.height}" for c in wl.cams}),
            "window": f"{wn}x{wn}", "sources": sorted({len(v.sources) for v in wl.input.views}),
            "megapixels_per_job": round(wl.pixels() / 1e6, 2),
            "iterations": f"{wl.photometric_iters} photometric + {wl.geometric_rounds}x{wl.geometric_iters} geometric",
            "math": math, "inputs": "8-bit gray images, seeded synthetic terrain",
            "l2": "inputs larger than L2 (24 f32 images + 1.2 GB of resident per-pixel state)",
            "parallelism": (f"one job's views sharded over {world} ranks" if shard_job else
                            f"{world} independent job(s), one per GPU")}


def bench_ours(args, rank, world, local):
    import torch
    from cumulus3d_b200 import _lib, densify, scenes
    from cumulus3d_b200.patchstereo import PatchMatchBackend, measure_fp32_peak

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    shard_job = world > 1 and args.shard_job
    wl = make_workload(args, rank, shard_job)
    if shard_job:
        from cumulus3d_b200.multigpu import shard_lpt, view_pixels
        mine = shard_lpt(view_pixels(wl.input), world)[rank]
    else:
        mine = list(range(len(wl.cams)))
    wn = 2 * wl.input.pm.window_radius // wl.input.pm.window_step + 1
    tuned = None
    args.tuning_was_auto = args.tuning < 0
    if args.tuning < 0:  # autotune the half-step variant on a prefix of this job's views (outside the timed region)
        from cumulus3d_b200.autotune import tune
        tuned = tune(wl.input, local, args.math, views=mine)
        args.tuning = tuned["tuning"]
    be = PatchMatchBackend(local, math=args.math, tuning=args.tuning)
    fp32_peak = measure_fp32_peak(local)
    sess = be.begin(wl.input)
    stream = torch.cuda.ExternalStream(sess.stream(), device=local)
    exchange = None
    if shard_job:
        from cumulus3d_b200.multigpu import SnapshotExchange
        exchange = SnapshotExchange(sess, wl.input, world, rank)

    def step():
        if exchange is None:  # one CUDA-graph launch per step (captured during the first warm-up step)
            sess.schedule_resident(mine, wl.photometric_iters, wl.geometric_rounds, wl.geometric_iters,
                                   graph=not args.no_graph)
        else:
            exchange.schedule(mine, wl.photometric_iters, wl.geometric_rounds, wl.geometric_iters)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        sess.synchronize()

    sess.set_profiling(True)  # before warm-up, so the captured graph carries the per-launch timing events
    for _ in range(args.warmup):
        step()
    barrier()
    sess.reset_stats()
    launches0 = sess.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        sess.synchronize()
        e1.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    launches = sess.launch_count() - launches0
    half = sess.kernel_stats(_lib.PS_KERNEL_HALF)
    ev = sess.kernel_stats(_lib.PS_KERNEL_EVAL)
    fl = sess.kernel_stats(_lib.PS_KERNEL_FILTER)
    sess.set_profiling(False)
    # whole-job time: max over ranks
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    views_total = len(wl.cams) * (1 if shard_job else world)
    iters = wl.iterations()
    value = views_total / (ms_step / 1e3)
    mpix_iter = wl.pixels() * (1 if shard_job else world) * iters / 1e6 / (ms_step / 1e3)
    # roofline of the dominant kernel (half step): algorithmic FLOP = windows × WN² taps × 33 FLOP, per launch
    half_launch_ms = half["ms"] / max(half["launches"], 1)
    taps_per_launch = half["ncc_windows"] * wn * wn / max(half["launches"], 1)
    skipped_per_launch = half["skipped_windows"] / max(half["launches"], 1)
    achieved = taps_per_launch * FLOP_PER_TAP_CACHED / (half_launch_ms / 1e3) / 1e12
    # the same time over the windows the reference evaluates: the evaluated ones plus those the early exit skips
    achieved_all = (taps_per_launch + skipped_per_launch * wn * wn) * FLOP_PER_TAP_CACHED / (half_launch_ms / 1e3) / 1e12
    traffic = None
    data_stage = None
    try:
        with open(os.path.join(ROOT, "profiles", "k_half_traffic.json")) as f:
            tr = json.load(f)
        traffic = tr["bytes_per_window"] * half["ncc_windows"] / max(half["launches"], 1)
        ds = tr.get("l1_data_stage")
        if ds:  # the binding resource, from the ncu capture (not measured by this run)
            data_stage = {"resource": "L1 data stage (texture gathers + shared-memory loads)", "busy": ds["busy"],
                          "texture_pipe": ds["texture_pipe_busy"], "lsu_pipe": ds["lsu_pipe_busy"],
                          "source": "ncu capture of one 6-view launch, profiles/k_half_c2_drone.md"}
    except Exception:
        pass
    res = {
        "metric": "PatchStereo views/s (drone-scale workload, 1 B200 per rank)", "value": round(value, 3),
        "unit": "views/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 3), "higher_is_better": True, "scaling": "strong" if shard_job else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded terrain renderer, no dataset)",
        "config": bench_config(wl, world, shard_job, args.math),
        "kernel": {"tuning": args.tuning,
                   "autotune": None if tuned is None else {"half_ms": tuned["ms"], "cached": tuned["cached"]}},
        "mpix_iter_per_s": round(mpix_iter, 2),
        "roofline": {"bound": "fp32", "kernel": "k_half", "achieved": round(achieved, 3),
                     "peak": round(fp32_peak, 2), "unit": "TFLOP/s", "frac": round(achieved / fp32_peak, 4),
                     "peak_source": "measured FFMA loop on this GPU (ps_measure_fp32_peak)",
                     "flop_per_tap": FLOP_PER_TAP_CACHED, "taps_per_launch": round(taps_per_launch),
                     "launch_ms": round(half_launch_ms, 3), "traffic": traffic,
                     "skipped_windows_per_launch": round(skipped_per_launch),
                     "frac_all_windows": round(achieved_all / fp32_peak, 4),
                     "binding_resource": data_stage,
                     "note": "achieved counts the NCC windows evaluated; refinement windows of candidates whose partial "
                             "cost already reached the best cost are skipped (same result), and frac_all_windows "
                             "counts them as the reference, which evaluates them, does"},
        "kernel_share": {"half": round(half["ms"], 2), "eval": round(ev["ms"], 2), "filter": round(fl["ms"], 2),
                         "timed_total": round(ms, 2)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    hbm = [hbm_used(local)]
    if not shard_job:
        res["fusion"] = fusion_stage(args, wl, sess, mine, check=rank == 0 and not args.no_check)
        hbm.append(hbm_used(local))
        if rank == 0 and not args.no_check:
            res["fp64_reeval"] = fp64_check(wl, sess, mine)
        res["neighbors"] = neighbors_stage(wl, sess, mine, local, check=rank == 0 and not args.no_check)
    if not args.no_learned and not shard_job:
        res["learned"] = learned_leg(args, wl, sess, stream, mine, value, ms_step, barrier, local)
        res["learned"]["fused_vs_plain"] = round(res["learned"]["fused_points"] / max(res["fusion"]["points"], 1), 4)
        hbm.append(hbm_used(local))
    if args.latency or args.workload == "c5":
        res["latency"] = view_latency(wl, sess, stream, mine)
    res["hbm_high_water_gb"] = round(max(hbm) / 1e9, 2)
    if not shard_job:
        res["fusion_all_options"] = fusion_options_stage(wl, sess, mine, check=rank == 0 and not args.no_check)
    if not args.no_c3 and args.workload == "c2" and not shard_job:
        try:  # an error in this leg is reported in the line instead of ending the run
            res["c3"] = c3_leg(args, local, fp32_peak, check=rank == 0 and not args.no_check)
        except Exception as e:  # noqa: BLE001
            res["c3"] = {"error": f"{type(e).__name__}: {e}"}
        try:  # an error in this leg is reported in the line instead of ending the run
            res["score_fusion"] = score_fusion_stage(wl, sess, mine, check=rank == 0 and not args.no_check)
        except Exception as e:  # noqa: BLE001
            res["score_fusion"] = {"error": f"{type(e).__name__}: {e}"}
    sess.close()
    # ---- e2e through the host-buffer C ABI (session begin uploads the images) ----
    if not args.no_e2e:
        res["e2e"] = e2e_leg(args, wl, be, mine, world, rank, local, exchange is not None, views_total)
    if rank == 0 and not args.no_cpu:
        res["cpu_baseline"] = cpu_baseline(wl, args)
    if exchange is not None:
        exchange.close()
    be.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return res


def c3_leg(args, local, fp32_peak, check=True, subset_per_size=2):
    """The batched uneven workload (64 views of 4 sizes from 4 terrains, 2-8 sources each) in one session: one
    warm-up schedule (graph capture), one timed schedule (CUDA events on the session stream), the half step's
    roofline, and a bitwise check of the ragged batching: a subset with `subset_per_size` views of every size runs
    once with all views in each launch and once with one view per launch, in fresh sessions; the maps must agree."""
    import torch
    from cumulus3d_b200 import _lib, scenes
    from cumulus3d_b200.patchstereo import PatchMatchBackend
    t0 = time.time()
    wl = scenes.workload_c3(seed=3)
    gen_s = time.time() - t0
    tuning = args.tuning
    tuned = None
    if getattr(args, "c3_tuning", -1) >= 0:
        tuning = args.c3_tuning
    elif args.tuning_was_auto:
        from cumulus3d_b200.autotune import tune
        tuned = tune(wl.input, local, args.math)
        tuning = tuned["tuning"]
    views = list(range(len(wl.cams)))
    wn = 2 * wl.input.pm.window_radius // wl.input.pm.window_step + 1
    be = PatchMatchBackend(local, math=args.math, tuning=tuning)
    sess = be.begin(wl.input)
    stream = torch.cuda.ExternalStream(sess.stream(), device=local)
    sess.set_profiling(True)
    run = lambda: sess.schedule_resident(views, wl.photometric_iters, wl.geometric_rounds, wl.geometric_iters)
    run()
    sess.synchronize()
    sess.reset_stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run()
    e1.record(stream)
    sess.synchronize()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    half = sess.kernel_stats(_lib.PS_KERNEL_HALF)
    sess.close()
    half_ms = half["ms"] / max(half["launches"], 1)
    taps = half["ncc_windows"] * wn * wn / max(half["launches"], 1)
    skipped = half["skipped_windows"] / max(half["launches"], 1)
    achieved = taps * FLOP_PER_TAP_CACHED / (half_ms / 1e3) / 1e12
    achieved_all = (taps + skipped * wn * wn) * FLOP_PER_TAP_CACHED / (half_ms / 1e3) / 1e12
    res = {"workload": wl.name, "views": len(views), "megapixels": round(wl.pixels() / 1e6, 2),
           "sizes": sorted({f"{c.width}x{c.height}" for c in wl.cams}),
           "sources": sorted({len(v.sources) for v in wl.input.views}),
           "iterations": f"{wl.photometric_iters} photometric + {wl.geometric_rounds}x{wl.geometric_iters} geometric",
           "value": round(len(views) / (ms / 1e3), 3), "unit": "views/s", "ms_per_step": round(ms, 2),
           "timed_steps": 1, "warmup": 1, "tuning": tuning,
           "autotune": None if tuned is None else {"half_ms": tuned["ms"], "cached": tuned["cached"], "key": tuned["key"]},
           "roofline": {"bound": "fp32", "kernel": "k_half", "achieved": round(achieved, 3), "peak": round(fp32_peak, 2),
                        "unit": "TFLOP/s", "frac": round(achieved / fp32_peak, 4), "launch_ms": round(half_ms, 3),
                        "frac_all_windows": round(achieved_all / fp32_peak, 4)},
           "scene_s": round(gen_s, 1)}
    if check:
        sizes = {}
        for v in views:
            sizes.setdefault((wl.cams[v].width, wl.cams[v].height), []).append(v)
        sub = sorted(v for vs in sizes.values() for v in vs[:subset_per_size])
        maps = []
        for mb in (64, 1):
            b2 = PatchMatchBackend(local, math=args.math, tuning=tuning, max_batch=mb)
            with b2.begin(wl.input) as s2:
                s2.schedule_resident(sub, wl.photometric_iters, wl.geometric_rounds, wl.geometric_iters)
                maps.append(s2.readout_download(0, sub))
            b2.close()
        equal = all(np.array_equal(a.depth, b.depth) and np.array_equal(a.normal, b.normal) and
                    np.array_equal(a.cost, b.cost) for a, b in zip(*maps))
        res["batch_check"] = {"views": sub, "equal": bool(equal),
                              "what": "the subset batched into every launch vs one view per launch (max_batch 1), "
                                      "fresh sessions, depth/normal/cost bitwise"}
    be.close()
    return res


def hbm_used(device):
    """Device memory in use (all allocations on the GPU, from cudaMemGetInfo)."""
    import torch
    free, total = torch.cuda.mem_get_info(device)
    return total - free


def fp64_check(wl, sess, mine):
    """FP64 re-evaluation of the final hypotheses of the first view: the engine's FP32 top-K photometric cost of the
    post-processed planes (ps_evaluate) against the oracle's binary64 restatement of the same cost."""
    from cumulus3d_b200.patchstereo import ViewState
    from oracle import oracle
    v = mine[0]
    st = sess.readout_download(0, [v])
    f32 = sess.evaluate(0, [v], st)[0].astype(np.float64)
    t0 = time.perf_counter()
    f64 = oracle.reeval_f64(wl.input, 0, [v], st)[0]
    dt = time.perf_counter() - t0
    m = st[0].depth > 0
    e = np.abs(f32 - f64)[m]
    flip = e >= 0.1  # a discrete test (centre inside the source image, variance floor) decided differently
    return {"view": v, "pixels": int(m.sum()), "max_abs_cost_err": float(e.max()) if e.size else None,
            "max_abs_cost_err_continuous": float(e[~flip].max()) if (~flip).any() else None,
            "decision_flips": int(flip.sum()),
            "mean_abs_cost_err": float(e.mean()) if e.size else None,
            "p99_abs_cost_err": float(np.percentile(e, 99)) if e.size else None,
            "frac_err_above_1e-3": float((e > 1e-3).mean()) if e.size else None, "oracle_s": round(dt, 2),
            "what": "top-K photometric cost (1 - NCC) of the final planes: FP32 engine vs FP64 CPU re-evaluation"}


def view_latency(wl, sess, stream, mine):
    """Latency of one view's photometric run alone on the GPU (run start + the workload's photometric iterations),
    CUDA-event timed per view: p50 / p99 over the job's views.  (In the batched schedule every view completes with the
    job.)"""
    import torch
    from cumulus3d_b200.patchstereo import RunParams
    ms = []
    for v in mine:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sess.run_resident([v], RunParams(0, False, True, wl.photometric_iters, 1))
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return {"p50_ms": round(float(np.percentile(ms, 50)), 2), "p99_ms": round(float(np.percentile(ms, 99)), 2),
            "views": len(ms), "what": f"one view, run start + {wl.photometric_iters} photometric iterations"}


def fusion_stage(args, wl, sess, mine, check=True, label="plain"):
    """Readout -> speckle removal -> consistency fusion (min 3 agreeing views) on the resident maps of the last step;
    with `check`, the CPU oracle fuses the same maps and must give the same point count."""
    import torch
    from cumulus3d_b200 import fusion
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src)
    prm = fusion.default_fusion(3)
    sess.readout_resident(mine, download=False)
    sess.synchronize()
    t0 = time.perf_counter()
    removed = sess.postprocess_resident(0, mine)
    n = sess.fuse_resident(0, mine, fc, prm)
    dt = time.perf_counter() - t0
    out = {"points": n, "speckle_pixels_removed": removed, "ms": round(dt * 1e3, 2),
           "params": "speckles (rel 0.02, area 2e-4, keep 0.2); consistency fusion min 3 views, 12 overlap views, "
                     "1 % depth, 2 px, 10 deg, inverse-variance weights"}
    if check:
        from oracle import oracle
        st = sess.readout_download(0, mine)
        t1 = time.perf_counter()
        from cumulus3d_b200 import scenes
        imgs = [scenes.unit_plane(kv.levels[0].pixels) if kv.levels[0].pixels.dtype == np.uint8
                else kv.levels[0].pixels for kv in wl.input.views]  # the f32 planes the engine computes with
        ref = oracle.fuse(fc, [x.depth for x in st], [x.normal for x in st], [x.cost for x in st], imgs, mine, prm)
        out["oracle_points"] = len(ref)
        out["oracle_s"] = round(time.perf_counter() - t1, 2)
        out["oracle_cores"] = os.cpu_count() or 1
    return out


def fusion_options_stage(wl, sess, mine, check=True, check_views=6):
    """Every post-processing and fusion option of the reference at once on the final maps: speckle removal, hole
    filling, consistency fusion with the second pass of leftover pixels, the visibility filter (8 views, 2 violations,
    1 %) and one smoothing pass, timed through the C ABI over all views after one untimed fusion with the same
    options.  With `check`, the device fuses the first
    `check_views` views again and the CPU oracle must give the same cloud bit for bit."""
    from cumulus3d_b200 import fusion
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src)
    post = fusion.default_post()
    post.fill_holes = 1
    prm = fusion.default_fusion(3)
    prm.residual = 2
    prm.visibility_check_views, prm.visibility_min_violations, prm.visibility_tau = 8, 2, 0.01
    prm.smooth_iterations = 1
    ks = np.array([c.k for c in wl.cams], np.float64)
    sess.readout_resident(mine, download=False)
    sess.fuse_resident(0, mine, fc, prm)  # warm-up (kernel loading, memory pool growth), untimed
    sess.readout_resident(mine, download=False)
    sess.synchronize()
    t0 = time.perf_counter()
    removed, filled = sess.postprocess_resident(0, mine, post, intrinsics=ks, filled=True)
    n = sess.fuse_resident(0, mine, fc, prm)
    dt = time.perf_counter() - t0
    out = {"points": n, "second_pass_points": sess.fused_residual,
           "visibility_removed": sess.fused_visibility_removed, "speckle_pixels_removed": removed,
           "pixels_filled": filled, "ms": round(dt * 1e3, 2),
           "params": "speckles and hole filling (PostParams defaults, fill on); consistency fusion min 3 views with "
                     "the second pass (ResidualParams defaults); visibility filter 8 views / 2 violations / 1 %; "
                     "1 smoothing pass (SmoothParams defaults)"}
    if check:
        from oracle import oracle
        from cumulus3d_b200 import scenes
        sub = list(mine[:check_views])
        n_sub = sess.fuse_resident(0, sub, fc, prm)
        got = sess.fused_points()
        st = sess.readout_download(0, mine)
        imgs = [scenes.unit_plane(kv.levels[0].pixels) if kv.levels[0].pixels.dtype == np.uint8
                else kv.levels[0].pixels for kv in wl.input.views]
        t1 = time.perf_counter()
        ref = oracle.fuse(fc, [x.depth for x in st], [x.normal for x in st], [x.cost for x in st], imgs, sub, prm)
        out["check"] = {"views": len(sub), "points": n_sub, "oracle_points": len(ref),
                        "oracle_s": round(time.perf_counter() - t1, 2),
                        "equal": bool(len(ref) == n_sub and np.array_equal(ref.keys, got.keys)
                                      and np.array_equal(ref.positions, got.positions)
                                      and np.array_equal(ref.normals, got.normals))}
    return out


def score_fusion_stage(wl, sess, mine, check=True, check_views=6):
    """Score fusion (fuse_scored, ScoreFusionOptions defaults: tau 2, λ 1, mark_used) of the final maps through the C
    ABI over all views, after one untimed run; with `check`, the device fuses the first `check_views` views again and
    the CPU oracle must give the same cloud bit for bit."""
    from cumulus3d_b200 import fusion
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src)
    prm = fusion.default_score_fusion()
    sess.readout_resident(mine, download=False)
    sess.postprocess_resident(0, mine)
    sess.fuse_scored_resident(0, mine, fc, prm)  # warm-up, untimed
    sess.synchronize()
    t0 = time.perf_counter()
    n = sess.fuse_scored_resident(0, mine, fc, prm)
    dt = time.perf_counter() - t0
    out = {"points": n, "ms": round(dt * 1e3, 2),
           "what": "candidates, claim rounds (mark_used) and the count, on the speckle-filtered final maps"}
    if check:
        from oracle import oracle
        from cumulus3d_b200 import scenes
        sub = list(mine[:check_views])
        n_sub = sess.fuse_scored_resident(0, sub, fc, prm)
        got = sess.fused_points()
        st = sess.readout_download(0, mine)
        imgs = [scenes.unit_plane(kv.levels[0].pixels) if kv.levels[0].pixels.dtype == np.uint8
                else kv.levels[0].pixels for kv in wl.input.views]
        t1 = time.perf_counter()
        ref = oracle.fuse_scored(fc, [x.depth for x in st], [x.normal for x in st], [x.cost for x in st], imgs, sub,
                                 prm)
        out["check"] = {"views": len(sub), "points": n_sub, "oracle_points": len(ref),
                        "oracle_s": round(time.perf_counter() - t1, 2),
                        "equal": bool(len(ref) == n_sub and np.array_equal(ref.keys, got.keys)
                                      and np.array_equal(ref.positions, got.positions)
                                      and np.array_equal(ref.normals, got.normals))}
    return out


def neighbors_stage(wl, sess, mine, local, check=True):
    """Neighbour views and depth ranges (ps_select_neighbors, NeighborOptions defaults) from sparse tracks built on the
    final filtered depth maps of the last step (seeded pixels back-projected and seen by every view whose depth
    agrees within 0.5 %); with `check`, the CPU oracle must give the same selections and ranges."""
    from cumulus3d_b200 import scenes
    from cumulus3d_b200.neighbors import NeighborParams, select_neighbors
    st = sess.readout_download(0, mine)
    depth = [x.depth for x in st]  # one map per view (views may differ in size)
    model = scenes.sparse_model([wl.cams[v] for v in mine], depth, 20000, seed=11)
    prm = NeighborParams()
    select_neighbors(model, prm, local)  # warm-up (module load)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        got = select_neighbors(model, prm, local)
        times.append(time.perf_counter() - t0)
    out = {"points": int(model.xyz.shape[0]), "observations": int(model.track_views.size),
           "ms": round(sorted(times)[1] * 1e3, 2),
           "what": "PairStats + select_all + depth_ranges on the GPU through the C ABI (host arrays in and out), "
                   "median of 3; NeighborOptions defaults (10 views, 1 deg)"}
    if check:
        from oracle import oracle
        t1 = time.perf_counter()
        ref = oracle.select_neighbors(model, prm)
        out["oracle_s"] = round(time.perf_counter() - t1, 2)
        out["equal"] = bool(ref.sources == got.sources and ref.depth_ranges == got.depth_ranges)
    return out


def net_flop_per_pixel():
    """Multiply-adds ×2 of one forward pass per full-resolution pixel (level l holds 4^-l of the pixels)."""
    from cumulus3d_b200.proposal import LAYERS
    level = (0, 0, 1, 1, 2, 2, 3, 3, 2, 1, 0, 0)
    return sum(2 * 9 * ci * co / 4 ** lv for (ci, co), lv in zip(LAYERS, level))


def learned_leg(args, wl, sess, stream, mine, plain_value, plain_ms, barrier, local):
    """The learned-init schedule on the same resident session: ps_propose (plane sweep + proposal network + decode)
    then the schedule with `--learned-iters` photometric iterations from the proposals (random init where the
    confidence is below `--learned-conf`), a geometric round of `--learned-geo-iters` iterations, filter and readout.  Timed like the plain step; accuracy is
    the agreement of the final filtered depth with the plain schedule's (within 1 % depth on the pixels the plain
    result keeps), next to the plain schedule's agreement with itself under another RNG seed and to a plain schedule
    shortened to the same iteration count."""
    import torch
    from cumulus3d_b200 import _lib, proposal

    proposal.set_conv_path(args.conv_path)
    net = proposal.ProposalNet(local, weights=args.weights or proposal.DEFAULT_WEIGHTS)
    k = args.learned_iters
    gi = args.learned_geo_iters
    # final depth maps of every view, flattened into one vector (views may differ in size)
    plain_depth = np.concatenate([o.depth.ravel() for o in sess.readout_resident(mine)])  # the last plain step's

    def depth():
        return np.concatenate([o.depth.ravel() for o in sess.readout_resident(mine)])

    def timed(fn, warm, steps):
        for _ in range(warm):
            fn()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        sess.synchronize()
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    def learned_step():
        sess.propose(net, 0, mine, args.learned_conf, count=False)
        sess.schedule_resident(mine, k, wl.geometric_rounds, gi, graph=not args.no_graph, proposal=True)

    sess.set_profiling(True)  # per-launch events for the sweep and network shares
    sess.reset_stats()
    ms_learned = timed(learned_step, args.warmup, args.steps)
    net_stats = sess.kernel_stats(_lib.PS_KERNEL_NET)
    sweep_stats = sess.kernel_stats(_lib.PS_KERNEL_SWEEP)
    sess.set_profiling(False)
    learned_depth = depth()
    learned_fused = fusion_stage(args, wl, sess, mine, check=False)["points"]
    ms_short = timed(lambda: sess.schedule_resident(mine, k, wl.geometric_rounds, gi, graph=not args.no_graph), 1, 2)
    short_depth = depth()
    short_fused = fusion_stage(args, wl, sess, mine, check=False)["points"]
    sess.schedule_resident(mine, wl.photometric_iters, wl.geometric_rounds, wl.geometric_iters, run_id_base=101,
                           graph=False)
    seed_depth = depth()
    ref_valid = plain_depth > 0

    def agree(d):
        return round(float((np.abs(d - plain_depth) <= 0.01 * plain_depth)[ref_valid].mean()), 4)

    steps_total = args.warmup + args.steps
    net_ms = net_stats["ms"] / max(net_stats["launches"], 1)
    pad_px = sum(((wl.cams[v].height + 7) // 8 * 8) * ((wl.cams[v].width + 7) // 8 * 8) for v in mine) / len(mine)
    flop = net_flop_per_pixel() * pad_px  # per view, averaged over the job's views
    peaks = _peaks()
    bf16_peak = peaks.get("bf16_tflops", 1590.0)
    achieved = flop / (net_ms / 1e3) / 1e12 if net_ms > 0 else float("nan")
    net.close()
    n = len(mine)
    return {
        "schedule": f"propose (plane sweep + network + decode) + {k} photometric from the proposal + "
                    f"{wl.geometric_rounds}x{gi} geometric + filter",
        "value": round(n / (ms_learned / 1e3), 3), "unit": "views/s", "ms_per_step": round(ms_learned, 2),
        "vs_plain": round(ms_step_ratio(plain_ms, ms_learned), 3),
        "propose_ms_per_view": round((net_stats["ms"] + sweep_stats["ms"]) / max(net_stats["launches"], 1), 3),
        "sweep_ms_per_view": round(sweep_stats["ms"] / max(sweep_stats["launches"], 1), 3),
        "net_ms_per_view": round(net_ms, 3),
        "accuracy": {"agree_with_plain": agree(learned_depth), "plain_other_seed": agree(seed_depth),
                     "coverage": round(float((learned_depth > 0).mean()), 4),
                     "coverage_plain": round(float(ref_valid.mean()), 4),
                     "definition": "fraction of the plain schedule's valid pixels whose final depth is within 1 % "
                                   "of it; the plain schedule rerun with another RNG seed sets the floor"},
        "fused_points": learned_fused,
        "plain_same_iterations": {"value": round(n / (ms_short / 1e3), 3), "ms_per_step": round(ms_short, 2),
                                  "agree_with_plain": agree(short_depth), "fused_points": short_fused,
                                  "coverage": round(float((short_depth > 0).mean()), 4)},
        "net_roofline": {"bound": "tensor", "kernel": "proposal network forward (12 conv layers, bf16; "
                         + {"auto": "tcgen05 for 64-128 output channels, mma.sync for 32",
                            "mma": "mma.sync only", "tcgen05": "tcgen05 only"}[args.conv_path] + ")",
                         "achieved": round(achieved, 2), "peak": bf16_peak, "unit": "TFLOP/s",
                         "frac": round(achieved / bf16_peak, 4), "peak_source": "MEASURED_PEAKS.json bf16_tflops "
                         "(measured)" if "bf16_tflops" in peaks else "fallback 1590",
                         "flop_per_view": round(flop / 1e9, 1), "unit_flop": "GFLOP"},
        "timed_steps": args.steps, "warmup": args.warmup, "steps_total": steps_total,
    }


def ms_step_ratio(plain_ms, other_ms):
    return plain_ms / other_ms


def e2e_leg(args, wl, be, mine, world, rank, local, multi, views_total):
    """The whole job through the host-buffer C ABI: ps_begin (image upload), the schedule with host states in and out
    of every call, then (one job per rank) speckle removal and consistency fusion (min 3 views) of the read-out maps
    and the download of the fused cloud."""
    import torch
    from cumulus3d_b200 import densify, fusion
    fc = fusion.FusionCams(wl.cams, [list(kv.sources) for kv in wl.input.views])
    prm = fusion.default_fusion(3)
    cloud_bytes = [0]

    def run_once():
        with be.begin(wl.input) as s:
            if multi:
                from cumulus3d_b200.multigpu import host_schedule_sharded
                host_schedule_sharded(s, wl.input, mine, wl.photometric_iters, wl.geometric_rounds,
                                      wl.geometric_iters, world, rank)
            else:
                densify.schedule_host(s, wl.input, mine, wl.photometric_iters, wl.geometric_rounds,
                                      wl.geometric_iters)
                s.readout_resident(mine, download=False)
                s.postprocess_resident(0, mine)
                s.fuse_resident(0, mine, fc, prm)
                cl = s.fused_points()
                cloud_bytes[0] = int(cl.positions.nbytes + cl.normals.nbytes + cl.colors.nbytes + cl.keys.nbytes +
                                     cl.vis_counts.nbytes + cl.vis.nbytes)
    for _ in range(max(1, min(args.warmup, 2))):
        run_once()
    torch.cuda.synchronize()
    steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(steps):
        run_once()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([dt], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt = float(t.item())
    npx = sum(wl.cams[v].width * wl.cams[v].height for v in mine)
    imgs = sum(c.width * c.height * 4 for c in wl.cams)
    runs = 1 + wl.geometric_rounds
    h2d = imgs + npx * (16 * wl.geometric_rounds + 4 * len(wl.cams) / max(len(mine), 1) * (wl.geometric_rounds + 1)
                        + 16)
    d2h = npx * (20 * runs + 1) + cloud_bytes[0]
    return {"value": round(views_total / dt, 3), "unit": "views/s", "ms_per_step": round(dt * 1e3, 2),
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "path": "ps_begin + ps_run/ps_filter with host ViewState buffers, then ps_postprocess_resident + "
                    "ps_fuse_resident + ps_fused_points (include/patchstereo.h)" if not multi else
                    "ps_begin + ps_run/ps_filter with host ViewState buffers (include/patchstereo.h)",
            "fused_cloud_bytes": cloud_bytes[0],
            "timer": "host wall clock around whole steps, max over ranks"}


def _snapshot_maps(wl, st0, gt):
    """Snapshot maps for view 0's geometric rounds: its own map, and its sources' ground truth when known (else view
    0's map again; the geometric term's cost does not depend on the values)."""
    maps = [None] * len(wl.cams)
    for v in range(len(wl.cams)):
        if gt is not None and v in gt:
            maps[v] = gt[v]
        elif (wl.cams[v].width, wl.cams[v].height) == (wl.cams[0].width, wl.cams[0].height):
            maps[v] = st0.depth
    maps[0] = st0.depth.copy()
    return maps


def cpu_sample(wl, threads=None, index=0, nbands=16, gt=None):
    """Times the CPU oracle on band `index` of `nbands` equal bands of full-width rows of view 0, through the whole
    per-view schedule: run start and the photometric iterations, the geometric rounds, the filter.  Scaled to the full
    view by pixel count.  The cost per row varies over the image (the top rows of the drone views cost about a third
    more than the average), so an estimate of the whole view averages the bands of a full cycle of indices.  Returns
    (per-view seconds, rows)."""
    from cumulus3d_b200.patchstereo import DepthSnapshot, RunParams, ViewState
    from oracle import oracle
    c = wl.cams[0]
    k = index % nbands
    rows = (c.height * k // nbands, c.height * (k + 1) // nbands)
    scale = c.height / (rows[1] - rows[0])
    st = [ViewState.new(c.width, c.height)]
    t0 = time.perf_counter()
    oracle.run(wl.input, [0], st, RunParams(0, False, True, wl.photometric_iters, 1), threads=threads, rows=rows)
    for r in range(wl.geometric_rounds):
        snap = DepthSnapshot(1 + r, 0, _snapshot_maps(wl, st[0], gt))
        oracle.run(wl.input, [0], st, RunParams(0, True, False, wl.geometric_iters, 2 + r), snap, threads=threads,
                   rows=rows)
    oracle.filter(wl.input, [0], st, DepthSnapshot(1 + wl.geometric_rounds, 0, _snapshot_maps(wl, st[0], gt)),
                  threads=threads, rows=rows)
    return (time.perf_counter() - t0) * scale, rows


def cpu_baseline(wl, args, nbands=16, picks=(1, 5, 9, 13)):
    cores = os.cpu_count() or 1
    est = [cpu_sample(wl, cores, k, nbands)[0] for k in picks]
    per_view = sum(est) / len(est)
    return {"value": round(1.0 / per_view, 5), "unit": "views/s", "cores": cores, "kind": "port",
            "sample": f"oracle (C++ restatement, OpenMP, all cores) on bands {list(picks)} of {nbands} equal bands of "
                      f"full-width rows of view 0, each through the whole per-view schedule ({wl.photometric_iters} "
                      f"photometric + {wl.geometric_rounds}x{wl.geometric_iters} geometric iterations + filter) and "
                      f"scaled by pixel count to a full view; the mean of the four",
            "mpix_iter_per_s": round(c_px(wl) * wl.iterations() / per_view / 1e6, 3)}


def c_px(wl):
    return wl.cams[0].width * wl.cams[0].height


def write_reference_workload(path: str) -> None:
    """Renders the drone-scale workload and stores what the reference arm needs (cameras, 8-bit images, sources, the
    ground-truth depth of view 0 and its sources) in an .npz.  Runs in a child process of the reference arm, so that
    the arm's own process maps only the CPU oracle's library."""
    from cumulus3d_b200 import scenes
    wl = scenes.workload_c2(with_gt=True)
    keep = [0] + list(wl.input.views[0].sources)
    np.savez(path, names=np.array([c.name for c in wl.cams]), k=np.array([c.k for c in wl.cams], np.float64),
             r=np.array([c.r for c in wl.cams]), t=np.array([c.t for c in wl.cams]),
             size=np.array([(c.width, c.height) for c in wl.cams]),
             gray=np.stack([kv.levels[0].pixels for kv in wl.input.views]),
             src_off=np.cumsum([0] + [len(kv.sources) for kv in wl.input.views]),
             src=np.array([j for kv in wl.input.views for j in kv.sources], np.int64),
             gt_views=np.array(keep), gt=np.stack([wl.gt_depth[v] for v in keep]),
             iters=np.array([wl.photometric_iters, wl.geometric_rounds, wl.geometric_iters]),
             window=np.array([wl.input.pm.window_radius, wl.input.pm.window_step]), name=np.array(wl.name))


def load_reference_workload(path: str):
    """The workload written by write_reference_workload, rebuilt without the renderer or the engine library."""
    from cumulus3d_b200 import scenes
    z = np.load(path)
    cams = [scenes.Camera(str(n), tuple(float(x) for x in k), r, t, int(sz[0]), int(sz[1]))
            for n, k, r, t, sz in zip(z["names"], z["k"], z["r"], z["t"], z["size"])]
    off = z["src_off"]
    src = [[int(j) for j in z["src"][off[i]:off[i + 1]]] for i in range(len(cams))]
    inp = scenes.kernel_input(cams, list(z["gray"]), src, (25.0, 60.0), window_radius=int(z["window"][0]),
                              window_step=int(z["window"][1]))
    it = [int(x) for x in z["iters"]]
    wl = scenes.Workload(str(z["name"]), cams, None, None, None, inp, it[0], it[1], it[2])
    gt = {int(v): z["gt"][i] for i, v in enumerate(z["gt_views"])}
    return wl, gt


def cpu_whole_view(wl, gt, threads=None):
    """Times the CPU oracle on the whole of view 0 through its full per-view schedule: run start and the photometric
    iterations, the geometric rounds, the filter.  The snapshot holds view 0's own depth map and the ground truth of
    its sources (_snapshot_maps; their own maps would need their schedules first).  Returns seconds."""
    from cumulus3d_b200.patchstereo import DepthSnapshot, RunParams, ViewState
    from oracle import oracle
    c = wl.cams[0]
    st = [ViewState.new(c.width, c.height)]
    t0 = time.perf_counter()
    oracle.run(wl.input, [0], st, RunParams(0, False, True, wl.photometric_iters, 1), threads=threads)
    for r in range(wl.geometric_rounds):
        oracle.run(wl.input, [0], st, RunParams(0, True, False, wl.geometric_iters, 2 + r),
                   DepthSnapshot(1 + r, 0, _snapshot_maps(wl, st[0], gt)), threads=threads)
    oracle.filter(wl.input, [0], st, DepthSnapshot(1 + wl.geometric_rounds, 0, _snapshot_maps(wl, st[0], gt)),
                  threads=threads)
    return time.perf_counter() - t0


def bench_reference(args, rank, world):
    """The reference arm: the CPU oracle (the restatement of the reference's PatchStereo, all host cores) on the
    same workload and config.  Step i times band i mod 16 of full-width rows of view 0 (a sixteenth of its height)
    through the whole per-view schedule, scaled by pixel count, and the value is the mean of the steps' estimates
    (16 steps cover the view once); one whole view through the same schedule is timed once and reported beside it
    with their ratio."""
    if rank != 0:
        return None
    import tempfile
    tmp = tempfile.mkdtemp(prefix="ps_ref_")
    path = os.path.join(tmp, "workload.npz")
    subprocess.run([sys.executable, os.path.abspath(__file__), "--write-reference-workload", path], check=True)
    wl, gt = load_reference_workload(path)
    cores = os.cpu_count() or 1
    for i in range(args.warmup):
        cpu_sample(wl, cores, i, 64, gt=gt)
    per = []
    t0 = time.perf_counter()
    for i in range(args.steps):  # step i times band i mod 16; 16 steps cover the whole view once
        per.append(cpu_sample(wl, cores, i, 16, gt=gt)[0])
    wall = time.perf_counter() - t0
    per_view = statistics.fmean(per)
    whole = None if args.no_whole_view else cpu_whole_view(wl, gt, cores)
    value = 1.0 / per_view
    res = {"impl": "reference", "metric": "PatchStereo views/s (drone-scale workload, 1 B200 per rank)",
           "value": round(value, 5), "unit": "views/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(wall / args.steps * 1e3, 1), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded terrain renderer, no dataset)",
           "config": bench_config(wl, world, False, "parity"),
           "cpu_baseline": {"value": round(value, 5), "unit": "views/s", "cores": cores, "kind": "port",
                            "sample": "step i: the CPU oracle (all cores) on band i mod 16 of view 0's rows (a "
                                      "sixteenth of the height) through the whole per-view schedule (photometric "
                                      "iterations, geometric rounds, filter), scaled by pixel count; value = 1 / the "
                                      "mean of the steps' estimates; the reference ships no CPU PatchStereo and its "
                                      "Rust/CUDA code cannot be built here"},
           "e2e": {"value": round(value, 5), "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if whole is not None:
        res["whole_view"] = {"seconds": round(whole, 2), "views_per_s": round(1.0 / whole, 5),
                             "band_estimate_over_whole": round(value * whole, 3),
                             "what": "view 0 at full size through run start, the photometric iterations, the "
                                     "geometric rounds and the filter on all cores, timed once"}
    os.remove(path)
    os.rmdir(tmp)
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--math", default="parity", choices=["parity", "fast"])
    ap.add_argument("--tuning", type=int, default=-1, help="half-step variant (PS_TUNE_* flags); -1 = autotune")
    ap.add_argument("--shard-job", action="store_true", help="shard one job's views over the ranks (strong scaling)")
    ap.add_argument("--workload", default="c2", choices=["c2", "c1", "c3", "c5"],
                    help="c2 = the metric's drone-scale configuration (default); c1/c3/c5 = the other configurations")
    ap.add_argument("--latency", action="store_true", help="per-view latency p50/p99 (always on for c5)")
    ap.add_argument("--views", type=int, default=None,
                    help="first N views of the workload only (small profiling cases, not a bench line)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="issue the schedule's launches directly (no CUDA graph)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the CPU oracle checks (fused point count, FP64 re-evaluation)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-init schedule")
    ap.add_argument("--no-c3", action="store_true", help="skip the batched uneven (64 mixed views) leg")
    ap.add_argument("--c3-tuning", type=int, default=-1, help="half-step variant of the c3 leg; -1 = autotune")
    ap.add_argument("--weights", default=None, help="proposal network parameters (.npz; default: the committed ones)")
    ap.add_argument("--conv-path", default="auto", choices=["auto", "mma", "tcgen05"],
                    help="network convolution kernels (auto: tcgen05 for cout >= 64, mma.sync below)")
    ap.add_argument("--learned-geo-iters", type=int, default=1,
                    help="iterations of the learned schedule's geometric round (the plain schedule's is 2)")
    ap.add_argument("--learned-conf", type=float, default=0.15,
                    help="confidence threshold of the proposals (random init below it)")
    ap.add_argument("--learned-iters", type=int, default=2,
                    help="photometric iterations of the learned-init schedule")
    ap.add_argument("--no-whole-view", action="store_true",
                    help="reference arm: skip the single whole-view timing of the CPU oracle")
    ap.add_argument("--write-reference-workload", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.write_reference_workload:
        write_reference_workload(args.write_reference_workload)
        return
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_env()
    if args.impl == "reference":
        res = bench_reference(args, rank, world)
    else:
        res = bench_ours(args, rank, world, local)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
