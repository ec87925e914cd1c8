#!/usr/bin/env python3
"""Benchmark of the B200 render path on the headline workload.

Workload (default): NoShadows, 1920x1080, 1 spp, a 1,000,000-triangle soup (seed 0, centroids
U[-1,1]^3, edges lognormal(ln 0.005, 0.5), random orientation), one point light, the reference CLI's
camera, BVH accelerator (built on the device).  One step = one Renderer::renderFrame of that frame
(mrt_render).  The reference renders rows 0..1071 of a 1080-row image (block height 1080/16 = 67,
Renderer.cpp:20-21); the rays counted are the rays traced.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  Under torchrun (N > 1) every rank renders its own frame on its own
GPU (independent frames: weak scaling, no collective on the data path); the timing is the maximum
over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WIDTH, HEIGHT, N_TRI, SEED = 1920, 1080, 1_000_000, 0
METRIC = "Mrays/s @1 B200, batched+served vs plain GPU vs host CPU; p50/p99 job latency"
WORKLOAD = ("NoShadows 1920x1080 1 spp, 1,000,000-triangle soup seed 0, 1 point light, "
            "BVH built on the device")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        """Starts sampling and waits for the first sample: nvidia-smi's start-up can hold the driver
        for a moment, which must not fall inside the timed region."""
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 20 and os.path.getsize(self.path) == 0:
            time.sleep(0.05)
        self.first = 0
        return self

    def mark(self):
        """Only samples after this call count (the start of the timed region)."""
        try:
            self.first = sum(1 for _ in open(self.path))
        except OSError:
            self.first = 0

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.path is None or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for k, line in enumerate(open(self.path)):
            if k < self.first:
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.remove(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profiled_traffic_per_ray():
    """DRAM bytes per ray of the render kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "render_noshadows_soup_1080p.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_ray:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def make_scene():
    from mobileraytracer_b200 import scenes
    t0 = time.time()
    sc = scenes.triangle_soup(N_TRI, SEED, WIDTH, HEIGHT)
    log(f"scene generated in {time.time() - t0:.1f}s")
    return sc


def cpu_baseline(sc, opts, budget_s: float, threads: int, first: int = 0):
    """The reference's own CPU renderer (oracle/_ref, compiled from the reference sources with its
    release optimisation level) on a bounded sample of the frame: every `step`-th pixel."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc as O
    from mobileraytracer_b200 import capi
    kind = "reference"
    try:
        O.ref(fast=True)
    except Exception as e:  # the checker library was not built
        log(f"cpu baseline unavailable: {e}")
        return None
    total = WIDTH * HEIGHT
    # probe: a few rays per thread to estimate the rate
    probe_step = max(1, total // (threads * 4))
    _, n, tb, tr = O.ref_render_subset(sc, sc.camera, opts, capi.MRT_ACCEL_BVH, threads, first, probe_step, fast=True)
    rate = n / max(tr, 1e-6)
    step = max(1, int(total / max(1.0, rate * budget_s)))
    _, n, tb2, tr = O.ref_render_subset(sc, sc.camera, opts, capi.MRT_ACCEL_BVH, threads, first + 1, step, fast=True)
    return {"value": n / tr / 1e6, "unit": "Mrays/s", "cores": threads, "kind": kind,
            "sample": f"every {step}th pixel of the {WIDTH}x{HEIGHT} frame ({n} camera rays), reference BVH "
                      f"(build {tb:.2f}s), {threads} threads", "rays": n, "seconds": tr, "build_seconds": tb}


def run_reference(args):
    """--impl reference: the reference's own CPU implementation of the path on the host cores."""
    ws, rank, local = dist_info()
    if rank != 0:
        return
    from mobileraytracer_b200 import capi
    sc = make_scene()
    opts = capi.render_opts(shader=capi.MRT_SHADER_NOSHADOWS, width=WIDTH, height=HEIGHT, spp=1, spl=1)
    threads = os.cpu_count() or 1
    per_step = max(1.5, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc as O
    try:
        O.ref(fast=True)
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU library not built: {e}"}))
        return
    total = WIDTH * HEIGHT
    _, n, tb, tr = O.ref_render_subset(sc, sc.camera, opts, capi.MRT_ACCEL_BVH, threads, 0, max(1, total // (threads * 4)), fast=True)
    rate = n / max(tr, 1e-6)
    step = max(1, int(total / max(1.0, rate * per_step)))
    for w in range(args.warmup):
        O.ref_render_subset(sc, sc.camera, opts, capi.MRT_ACCEL_BVH, threads, w + 1, step, fast=True)
    rays, secs = 0, 0.0
    for k in range(args.steps):
        _, n, _, tr = O.ref_render_subset(sc, sc.camera, opts, capi.MRT_ACCEL_BVH, threads, args.warmup + 1 + k,
                                          step, fast=True)
        rays += n
        secs += tr
    value = rays / secs / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_per_step": f"every {step}th pixel", "accelerator": "reference BVH"},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "reference",
                         "sample": f"every {step}th pixel of the {WIDTH}x{HEIGHT} frame per step, reference BVH "
                                   f"(build {tb:.2f}s), {threads} threads"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


BATCH_WORKLOAD = ("256 PathTracer jobs (depth 6, Russian roulette beyond depth 3, 1 light sample), "
                  "job i = triangle soup of seed i with N log-uniform over [1e3, 2e6], 4 area-light quads of "
                  "emission 10, square image of side log-uniform over [128, 1024] (multiple of 16), spp uniform "
                  "over {1, 4, 16, 64}")


def _job_geometry(job):
    """(tri_abc) of one batched job; runs in a spawn pool before the GPU is touched."""
    from mobileraytracer_b200 import scenes
    return scenes._soup_geometry(job.n_triangles, job.seed)


def generate_jobs(jobs, workers: int):
    """Host scenes of the batched jobs, generated in parallel (spawn pool: no CUDA state is forked)."""
    import multiprocessing as mp
    from mobileraytracer_b200 import scenes
    t0 = time.time()
    with mp.get_context("spawn").Pool(max(1, workers)) as pool:
        geoms = pool.map(_job_geometry, jobs, chunksize=1)
    out = []
    for job, g in zip(jobs, geoms):
        s = scenes.Scene()
        s.tri_abc = g
        s.tri_material = np.zeros(job.n_triangles, np.int32)
        s.materials = [scenes._material(kd=(0.8, 0.8, 0.8))]
        s.lights = scenes._quad_lights(10.0)
        s.camera = scenes.cli_camera(job.side, job.side)
        out.append(s)
    log(f"{len(jobs)} job scenes ({sum(j.n_triangles for j in jobs)} triangles) generated in {time.time() - t0:.1f}s")
    return out


def job_opts(job, capi, spp_offset: int = 0, spp: int | None = None):
    return capi.render_opts(shader=capi.MRT_SHADER_PATHTRACER, width=job.side, height=job.side,
                            spp=job.spp if spp is None else spp, spl=1, depth_min=3, depth_max=6, seed=job.seed,
                            spp_offset=spp_offset)


def bench_batched(args):
    """The 256-job batch: the batched renderer against the plain one-job-per-launch renderer on the same job
    list.  One step = every job rendered once; value = rays traced / wall time of the step."""
    from mobileraytracer_b200 import scenes
    jobs = scenes.batched_jobs(args.jobs)
    host = generate_jobs(jobs, min(16, os.cpu_count() or 1))
    import torch
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import capi
    torch.cuda.set_device(0)
    ctx = m.Context(0)
    t0 = time.time()
    built = [m.Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST) for sc in host]
    build_s = time.time() - t0
    arena_bytes = sum(b.device_bytes() for b in built)
    opts = [job_opts(j, capi) for j in jobs]
    bm_plain = [torch.zeros(j.side * j.side, dtype=torch.int32, device="cuda") for j in jobs]
    bm_batch = [torch.zeros(j.side * j.side, dtype=torch.int32, device="cuda") for j in jobs]
    paths = sum(j.side * j.side * j.spp for j in jobs)

    def plain_step():
        rays = 0
        torch.cuda.synchronize()
        t = time.perf_counter()
        for k, j in enumerate(jobs):
            _, _, st = built[k].render(host[k].camera, opts[k], bitmap=bm_plain[k])
            rays += st.rays_closest + st.rays_shadow
        torch.cuda.synchronize()
        return rays, time.perf_counter() - t

    policy = {"smallest": capi.MRT_BATCH_SMALLEST_FIRST, "fifo": capi.MRT_BATCH_FIFO,
              "share": capi.MRT_BATCH_EQUAL_SHARE}[args.policy]
    batch = m.Batch(ctx, max_depth=6, max_spl=1, max_jobs=max(4096, len(jobs)), wave_roots=args.wave_roots,
                    policy=policy, pipelines=args.pipelines)

    def batch_step():
        s0 = batch.stats()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for k, j in enumerate(jobs):
            batch.submit(built[k], host[k].camera, opts[k], bm_batch[k])
        batch.run()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        batch.completed()
        s1 = batch.stats()
        return (s1.rays_closest + s1.rays_shadow) - (s0.rays_closest + s0.rays_shadow), dt, s1.busy_ms - s0.busy_ms

    clocks = ClockSampler(0).__enter__()
    for _ in range(args.warmup):
        batch_step()
    plain_step()
    clocks.mark()
    b_rays = b_time = b_busy = 0.0
    for _ in range(args.steps):
        r, dt, busy = batch_step()
        b_rays += r
        b_time += dt
        b_busy += busy
    p_rays = p_time = 0.0
    for _ in range(args.steps):
        r, dt = plain_step()
        p_rays += r
        p_time += dt
    clocks.__exit__(None, None, None)
    same = sum(int(torch.equal(a, b)) for a, b in zip(bm_plain, bm_batch))
    st = batch.stats()
    value = b_rays / b_time / 1e6
    plain_value = p_rays / p_time / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": b_time * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "jobs": len(jobs), "paths_per_step": paths,
                   "triangles": sum(j.n_triangles for j in jobs), "scene_device_bytes": arena_bytes,
                   "scene_build_seconds": build_s, "rays_per_step": b_rays / args.steps,
                   "l2": "inputs (scenes ~GBs) far larger than L2",
                   "policy": args.policy, "wave_roots": st.wave_roots, "block_threads": st.block_threads,
                   "blocks_per_sm": st.blocks_per_sm, "pipelines": st.pipelines, "autotuner_probes": st.autotuned,
                   "whole_path_waves": st.waves_paths,
                   "waves_per_step": st.waves / (args.warmup + args.steps),
                   "device_busy_fraction": b_busy / 1e3 / b_time},
        "plain": {"value": plain_value, "unit": "Mrays/s", "ms_per_step": p_time * 1e3 / args.steps,
                  "rays_per_step": p_rays / args.steps, "renderer": "mrt_render per job, device buffers"},
        "batched_over_plain": value / plain_value,
        "bitmaps_equal_plain": f"{same}/{len(jobs)}",
        "gpu_launches": None,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)
    batch.close()
    for b in built:
        b.close()
    ctx.close()


SERVE_WORKLOAD = ("Poisson stream of render requests, each drawn as a batched-workload job (PathTracer "
                  "depth 6, soup geometry from the 256-job pool, side log-uniform over [128, 1024], spp uniform "
                  "over {1, 4, 16, 64}); 20% re-render one of the last 64 new scenes with +16 spp progressive "
                  "accumulation; admission by device footprint")


def bench_served(args):
    """The request stream: the same requests served by the batched renderer (continuous batching) and by
    one mrt_render call per request; throughput, p50/p99 latency, offered vs achieved load."""
    from mobileraytracer_b200 import scenes
    from mobileraytracer_b200 import serve
    pool = scenes.batched_jobs(256)
    host = generate_jobs(pool, min(16, os.cpu_count() or 1))
    reqs = serve.request_stream(pool, duration_s=args.duration, rate=args.rate)
    offered_paths = sum(r.paths for r in reqs)
    log(f"{len(reqs)} requests over {args.duration}s ({sum(r.kind == 'rerender' for r in reqs)} re-renders), "
        f"{offered_paths / args.duration / 1e6:.1f} M paths/s offered")
    import torch
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import capi
    torch.cuda.set_device(0)
    budget = int(args.budget_gb * 1e9)
    bitmap_reserve = 8 << 30          # images of every scene served (kept for progressive re-renders)
    build_slack = 1 << 30             # tree-build scratch of the scene being built
    scene_budget = budget - bitmap_reserve - build_slack

    def pool_scene(r):
        return host[r.geometry]

    results = {}
    clocks = ClockSampler(0).__enter__()
    clocks.mark()
    for kind in ("plain", "batched"):
        ctx = m.Context(0)
        arena = m.Arena(0, scene_budget + build_slack)
        if kind == "batched":
            be = serve.BatchBackend(ctx, arena, pool_scene, dict(
                max_depth=6, max_spl=1, max_jobs=4096, wave_roots=args.wave_roots or (1 << 20),
                max_wave_roots=max(args.wave_roots, 1 << 20), block_threads=64, blocks_per_sm=16,
                pipelines=args.pipelines or 4))
        else:
            be = serve.PlainBackend(ctx, arena, pool_scene)
        loop = serve.ServeLoop(reqs, be, scene_budget)
        t = time.perf_counter()
        summary = loop.run()
        torch.cuda.synchronize()
        summary["wall_seconds"] = time.perf_counter() - t
        summary["rays"] = be.total_rays()
        summary["checksums"] = dict(be.checksums)
        summary["arena"] = arena.stats()
        be.close()
        ctx.close()
        arena.close()
        results[kind] = summary
        log(f"{kind}: {summary['wall_seconds']:.1f}s, p50 {summary['latency_p50_s']:.3f}s p99 "
            f"{summary['latency_p99_s']:.3f}s, {summary['rays'] / summary['wall_seconds'] / 1e6:.1f} Mrays/s")
    clocks.__exit__(None, None, None)
    same = sum(int(results["plain"]["checksums"][i] == results["batched"]["checksums"][i]) for i in range(len(reqs)))

    def summ(r):
        return {"Mrays_per_s": r["rays"] / r["wall_seconds"] / 1e6, "wall_seconds": r["wall_seconds"],
                "latency_p50_s": r["latency_p50_s"], "latency_p99_s": r["latency_p99_s"],
                "latency_mean_s": r["latency_mean_s"], "achieved_paths_per_s": offered_paths / r["wall_seconds"],
                "rays": r["rays"], "evictions": r["evictions"], "rebuilds_after_eviction": r["rebuilds_after_eviction"],
                "peak_scene_bytes": r["peak_scene_bytes"], "arena_peak_bytes": r["arena"]["peak"]}

    b, p = summ(results["batched"]), summ(results["plain"])
    line = {
        "metric": METRIC, "value": b["Mrays_per_s"], "unit": "Mrays/s", "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": b["wall_seconds"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": SERVE_WORKLOAD, "duration_s": args.duration, "rate_per_s": args.rate,
                   "requests": len(reqs), "rerenders": sum(r.kind == "rerender" for r in reqs),
                   "offered_paths_per_s": offered_paths / args.duration, "budget_bytes": budget,
                   "scene_budget_bytes": scene_budget, "bitmap_reserve_bytes": bitmap_reserve,
                   "build_slack_bytes": build_slack},
        "served": b, "plain": p, "served_over_plain": b["Mrays_per_s"] / p["Mrays_per_s"],
        "results_equal_plain": f"{same}/{len(reqs)}",
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


SCENE_WORKLOADS = {
    "cornell": ("Whitted 256x256, 1 spp (Constant 0.5 camera sampler), procedural Cornell box "
                "(10 wall + 24 box triangles, mirror sphere, 2 area-light triangles of emission 15), BVH"),
    "terrain": ("PathTracer 1024x1024, 64 spp HaltonSeq (camera, light and roulette), depth 6 with "
                "Russian roulette beyond depth 3, 512x512 fBm heightfield (524,288 triangles), 4 area-light quads "
                "of emission 10, fp32 sums"),
}


def scene_workload(name):
    from mobileraytracer_b200 import capi, scenes
    if name == "cornell":
        sc = scenes.cornell_box()
        opts = capi.render_opts(shader=capi.MRT_SHADER_WHITTED, width=256, height=256, spp=1, spl=1, seed=1)
    else:
        sc = scenes.heightfield(cells=512, seed=1)
        H = capi.MRT_SAMPLER_HALTON
        opts = capi.render_opts(shader=capi.MRT_SHADER_PATHTRACER, width=1024, height=1024, spp=64, spl=1,
                                pixel_sampler=H, light_sampler=H, rr_sampler=H, depth_min=3, depth_max=6, seed=1)
    return sc, opts


def bench_scene(args):
    """Configs 1 and 3: one step = one Renderer::renderFrame of the frame (mrt_render on device
    buffers); value = rays traced (camera + secondary + shadow) / device time."""
    import torch
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import capi
    sc, opts = scene_workload(args.workload)
    torch.cuda.set_device(0)
    ctx = m.Context(0)
    t0 = time.time()
    scene = m.Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    build_s = time.time() - t0
    w, h = opts.width, opts.height
    bitmap = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    accum = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream, device="cuda")

    def step():
        with torch.cuda.stream(stream):
            flush.fill_(1)   # evicts L2 (126 MB) before every step; not inside the timed events
        _, _, st = scene.render(sc.camera, opts, bitmap=bitmap, accum=accum)
        return st

    clocks = ClockSampler(0).__enter__()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks.mark()
    dev_ms = 0.0
    rays = paths = 0
    for _ in range(args.steps):
        st = step()
        dev_ms += st.device_ms
        rays += st.rays_closest + st.rays_shadow
        paths += st.paths
    torch.cuda.synchronize()
    clocks.__exit__(None, None, None)
    value = rays / (dev_ms / 1e3) / 1e6
    rays_per_path = rays / paths
    # end to end: host bitmap and sums (pinned) in and out through the C ABI
    host_bm = torch.zeros((h, w), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    host_acc = torch.zeros((h, w, 4), dtype=torch.float32).pin_memory().numpy()
    scene.render(sc.camera, opts, bitmap=host_bm, accum=host_acc)
    n_e2e = max(1, min(args.e2e_steps, args.steps))
    t1 = time.perf_counter()
    for _ in range(n_e2e):
        scene.render(sc.camera, opts, bitmap=host_bm, accum=host_acc)
    e2e_s = (time.perf_counter() - t1) / n_e2e
    cpu = None
    if not args.no_cpu_baseline:
        cpu = scene_cpu_baseline(sc, opts, rays_per_path, args.cpu_budget)
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": SCENE_WORKLOADS[args.workload], "rays_per_step": rays / args.steps,
                   "paths_per_step": paths / args.steps, "rays_per_path": rays_per_path,
                   "samples_per_s": paths / (dev_ms / 1e3), "bvh_build_seconds": build_s,
                   "l2": "flushed before every step (512 MiB write outside the timed events)"},
        "e2e": {"value": rays / args.steps / e2e_s / 1e6, "unit": "Mrays/s",
                "h2d_bytes_per_step": host_bm.nbytes - 4 * w * 16 * (h // 16) + host_acc.nbytes,
                "d2h_bytes_per_step": host_bm.nbytes + host_acc.nbytes},
        "gpu_launches": None, "roofline": None, "clocks": clocks.summary(), "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()


def bench_raster(args):
    """The raster preview of the 1920x1080 frame's soup (1,000,000 triangles, 1920x1080): one step = one
    mrt_raster_preview on a device bitmap; value = scene triangles / device time (Mtris/s)."""
    import torch
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import scenes
    w, h = 1920, 1080
    sc = scenes.triangle_soup(1_000_000, 0, w, h)
    torch.cuda.set_device(0)
    ctx = m.Context(0)
    scene = m.Scene(ctx, sc)
    bitmap = torch.zeros((h, w), dtype=torch.int32, device="cuda")
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream, device="cuda")

    def step():
        with torch.cuda.stream(stream):
            flush.fill_(1)   # evicts L2 before every step; not inside the timed events
        return scene.raster_preview(sc.camera, w, h, bitmap=bitmap)[1]

    clocks = ClockSampler(0).__enter__()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks.mark()
    dev_ms, st = 0.0, None
    for _ in range(args.steps):
        st = step()
        dev_ms += st.device_ms
    torch.cuda.synchronize()
    clocks.__exit__(None, None, None)
    ms = dev_ms / args.steps
    covered = int((bitmap != 0).sum().item())
    # algorithmic bytes: 48 per triangle (A, AB, AC records), per pixel 8 (depth-key clear) + 8 (key
    # read) + 4 (bitmap write), 8 per covered sample (the atomicMin), 4 per drawn pixel (material id)
    algo = 48 * sc.n_triangles + 20 * w * h + 8 * st.fragments + 4 * covered
    peak, peak_src = measured_peak()
    achieved = algo / (ms / 1e3) / 1e9
    host_bm = torch.zeros((h, w), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    scene.raster_preview(sc.camera, w, h, bitmap=host_bm)
    n_e2e = max(1, min(args.e2e_steps, args.steps))
    t1 = time.perf_counter()
    for _ in range(n_e2e):
        scene.raster_preview(sc.camera, w, h, bitmap=host_bm)
    e2e_s = (time.perf_counter() - t1) / n_e2e
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import orc as O
        try:
            n, t = 0, 0.0
            while t < min(args.cpu_budget, 10.0):
                t0 = time.perf_counter()
                O.raster_preview(sc, sc.camera, w, h)
                t += time.perf_counter() - t0
                n += 1
            cpu = {"value": n * sc.n_triangles / t / 1e6, "unit": "Mtris/s", "cores": 1, "kind": "port",
                   "sample": f"{n} whole previews by the oracle's serial restatement (the reference draws with "
                             f"OpenGL ES, unavailable here)"}
        except Exception as e:   # the checker library was not built
            log(f"cpu baseline unavailable: {e}")
    line = {
        "metric": METRIC, "value": sc.n_triangles / (ms / 1e3) / 1e6, "unit": "Mtris/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "raster preview (MainRenderer.copyFrame) of the 1,000,000-triangle soup seed 0, "
                               "1920x1080, the CLI camera", "triangles": sc.n_triangles, "drawn": st.drawn,
                   "fragments": st.fragments, "covered_pixels": covered,
                   "l2": "flushed before every step (512 MiB write outside the timed events)"},
        "e2e": {"value": sc.n_triangles / e2e_s / 1e6, "unit": "Mtris/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": host_bm.nbytes},
        "gpu_launches": 3 * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": None, "algorithmic_bytes_per_launch": algo,
                     "kernel": "k_raster_tris + k_raster_big + k_raster_resolve (+ key clear)"},
        "clocks": clocks.summary(), "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()


def scene_cpu_baseline(sc, opts, rays_per_path: float, budget_s: float):
    """The reference's CPU renderer (oracle/_ref, its release optimisation level) on the host cores.
    It traces but does not count rays, so its Mrays/s is its camera paths per second times the rays
    per path the device counted on the same frame."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc as O
    from mobileraytracer_b200 import capi
    threads = os.cpu_count() or 1
    try:
        O.ref(fast=True)
    except Exception as e:  # the checker library was not built
        log(f"cpu baseline unavailable: {e}")
        return None
    if opts.width * opts.height * opts.spp <= 1 << 17:   # small frame: whole frames, repeated
        n, t = 0, 0.0
        while t < budget_s / 4:
            _, _, tr = O.ref_render(sc, sc.camera, opts, capi.MRT_ACCEL_BVH, threads, fast=True)
            n += 1
            t += tr
        paths = n * opts.width * 16 * (opts.height // 16) * opts.spp
        sample = f"{n} whole {opts.width}x{opts.height} frames, reference BVH, {threads} threads"
    else:                                                # one sample of every step-th pixel
        total = opts.width * opts.height
        one = capi.render_opts(shader=opts.shader, width=opts.width, height=opts.height, spp=1, spl=opts.spl,
                               pixel_sampler=opts.pixel_sampler, light_sampler=opts.light_sampler,
                               rr_sampler=opts.rr_sampler, depth_min=opts.depth_min, depth_max=opts.depth_max,
                               seed=opts.seed)
        _, n0, _, tr0 = O.ref_render_subset(sc, sc.camera, one, capi.MRT_ACCEL_BVH, threads, 0,
                                            max(1, total // (threads * 16)))
        step = max(1, int(total / max(1.0, n0 / max(tr0, 1e-6) * budget_s)))
        _, paths, _, t = O.ref_render_subset(sc, sc.camera, one, capi.MRT_ACCEL_BVH, threads, 1, step)
        sample = (f"sample 0 of every {step}th pixel of the {opts.width}x{opts.height} frame ({paths} camera paths), "
                  f"reference BVH and samplers, {threads} threads")
    return {"value": paths * rays_per_path / t / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "sample": sample, "paths_per_s": paths / t, "rays_per_path_assumed": rays_per_path}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 200 frames, or 1 batch)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of reference CPU work for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="frame", choices=["frame", "cornell", "terrain", "batched", "served", "raster"],
                    help="frame: the 1920x1080 NoShadows frame (default); cornell / terrain: the Whitted and "
                         "PathTracer frames; batched: the 256-job batch; served: the request stream; raster: the "
                         "raster preview of the frame's soup")
    ap.add_argument("--duration", type=float, default=120.0, help="served: seconds of arrivals")
    ap.add_argument("--rate", type=float, default=50.0, help="served: arrivals per second")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="served: device footprint budget")
    ap.add_argument("--pipelines", type=int, default=0, help="batched/served: waves in flight (0: autotuned / 4)")
    ap.add_argument("--jobs", type=int, default=256, help="batched: jobs in the list")
    ap.add_argument("--wave-roots", type=int, default=0, help="batched: camera paths per wave (0: autotuned)")
    ap.add_argument("--policy", default="smallest", choices=["smallest", "fifo", "share"],
                    help="batched: which jobs fill a wave")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = {"batched": 1, "terrain": 3}.get(args.workload, 200)
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batched":
        bench_batched(args)
        return
    if args.workload == "served":
        bench_served(args)
        return
    if args.workload == "raster":
        bench_raster(args)
        return
    if args.workload in SCENE_WORKLOADS:
        bench_scene(args)
        return

    import torch
    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import camera as mcam
    from mobileraytracer_b200 import capi

    sc = make_scene()
    ctx = m.Context(local)
    t0 = time.time()
    scene = m.Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    build_s = time.time() - t0
    opts = capi.render_opts(shader=capi.MRT_SHADER_NOSHADOWS, width=WIDTH, height=HEIGHT, spp=1, spl=1)
    bitmap = torch.zeros(WIDTH * HEIGHT, dtype=torch.int32, device=f"cuda:{local}")
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")

    def step():
        with torch.cuda.stream(stream):
            flush.fill_(1)   # evicts L2 (126 MB) before every step; not inside the timed events
        _, _, st = scene.render(sc.camera, opts, bitmap=bitmap)
        return st

    clocks = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
        step()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    dev_ms, rays = 0.0, 0
    clocks.mark()
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        st = step()
        dev_ms += st.device_ms
        rays += st.rays_closest
    torch.cuda.synchronize()
    clocks.__exit__(None, None, None)
    wall = time.perf_counter() - wall0
    if ws > 1:
        t = torch.tensor([dev_ms], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        dev_ms = float(t.item())
        torch.distributed.barrier()
    rays_per_step = rays // args.steps
    value = rays_per_step * args.steps * ws / (dev_ms / 1e3) / 1e6
    ms_per_step = dev_ms / args.steps

    # end to end through the C ABI with host buffers: pinned bitmap in, render, bitmap out
    host_bm = torch.zeros(WIDTH * HEIGHT, dtype=torch.int32).pin_memory()
    host_np = host_bm.numpy()
    scene.render(sc.camera, opts, bitmap=host_np)
    e2e_t = 0.0
    e2e_n = max(1, min(args.e2e_steps, args.steps))
    for _ in range(e2e_n):
        t1 = time.perf_counter()
        scene.render(sc.camera, opts, bitmap=host_np)
        e2e_t += time.perf_counter() - t1
    e2e_value = rays_per_step * e2e_n * ws / e2e_t / 1e6
    bm_bytes = WIDTH * HEIGHT * 4

    # roofline: algorithmic bytes per launch from the counting replay over the same camera rays
    rays_np = mcam.primary_rays(sc.camera, WIDTH, HEIGHT, pixels=np.arange(WIDTH * 16 * (HEIGHT // 16)))
    nodes, tris = scene.trace_counts(rays_np)
    hits = scene.trace_closest(rays_np)
    n_hit = int(np.sum((hits["id"] >> 30) == capi.MRT_PRIM_TRIANGLE))
    alg_bytes = 8 * len(rays_np) + 32 * int(nodes.sum(dtype=np.int64)) + 48 * int(tris.sum(dtype=np.int64)) + 76 * n_hit
    achieved = alg_bytes / (ms_per_step / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    tpr = profiled_traffic_per_ray()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_kind, "traffic": (tpr * len(rays_np)) if tpr else None,
            "algorithmic_bytes_per_launch": alg_bytes, "bytes_per_ray": alg_bytes / len(rays_np),
            "node_records_per_ray": float(nodes.mean()), "tri_records_per_ray": float(tris.mean()),
            "kernel": "k_render_noshadows_fast (persistent)"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sc, opts, args.cpu_budget, os.cpu_count() or 1)
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rays_per_step": rays_per_step, "rows_rendered": 16 * (HEIGHT // 16),
                   "l2": "flushed before every step (512 MiB write outside the timed events)",
                   "bvh_build_seconds": build_s, "wall_seconds_timed_loop": wall, "parallelism": f"replicas x{ws}"},
        # in: the bitmap rows the block schedule leaves alone (a first pass overwrites the rest without
        # reading it), camera and options; out: the whole bitmap
        "e2e": {"value": e2e_value, "unit": "Mrays/s",
                "h2d_bytes_per_step": bm_bytes - 4 * WIDTH * 16 * (HEIGHT // 16) + 64 + 100,
                "d2h_bytes_per_step": bm_bytes},
        "gpu_launches": args.steps,
        "roofline": roof,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
