#!/usr/bin/env python3
"""Benchmark of the B200 render path: the headline frame and every configuration of the metric.

Headline (the line's `value`): NoShadows, 1920x1080, 1 spp, a 1,000,000-triangle soup (seed 0,
centroids U[-1,1]^3, edges lognormal(ln 0.005, 0.5), random orientation), one point light, the
reference CLI's camera, FAST BVH built on the device.  One step = one Renderer::renderFrame of that
frame (mrt_render).  The reference renders rows 0..1071 of a 1080-row image (block height 1080/16 =
67, Renderer.cpp:20-21); the rays counted are the rays traced.

The same line carries, under "configs", every other configuration of the metric measured in the same
run: the soup frame on the RegularGrid (G = 128 by the reference's sizing rule, and G = 100 =
cbrt(N) with linear cell indexing), the Whitted Cornell box, the PathTracer terrain, the 256-job
batch against one mrt_render per job, and a served request stream (p50/p99 latency) against one
render per request.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]

Prints one JSON line (rank 0).  Under torchrun (N > 1) every rank renders its own frames on its own
GPU (independent frames: weak scaling, no collective on the data path), batched jobs and served
requests are split across ranks; timings are the maximum over ranks.
"""
from __future__ import annotations

import argparse
import hashlib
import json
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
FRAME = "NoShadows 1920x1080 1 spp, 1,000,000-triangle soup seed 0, 1 point light, the CLI camera"
WORKLOAD = FRAME + ", FAST BVH built on the device"
REF_WORKLOAD = FRAME + ", the reference's BVH (BVH<Triangle>, top-down SAH) built on the host"
PROFILE = os.path.join(ROOT, "profiles", "ns_trace_soup_1080p.md")
GRID_PROFILE = os.path.join(ROOT, "profiles", "ns_trace_grid_soup_1080p.md")
FAST_NODE_BYTES = 128  # bytes of one 8-wide node, the unit of the FAST tree's counting replay


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    """One process per GPU.  Collectives are used only for timing (max over ranks), sums of counts
    and gathering per-request records; every rank calls them in the same order."""

    def __init__(self):
        self.ws, self.rank, self.local = dist_info()
        import torch
        torch.cuda.set_device(self.local)
        self.device = f"cuda:{self.local}"
        if self.ws > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                    device_id=torch.device("cuda", self.local))

    def _reduce(self, x: float, op: str) -> float:
        if self.ws == 1:
            return float(x)
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(x)], device=self.device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, "max")

    def sum(self, x: float) -> float:
        return self._reduce(x, "sum")

    def gather(self, obj) -> list:
        if self.ws == 1:
            return [obj]
        import torch.distributed as dist
        out = [None] * self.ws
        dist.all_gather_object(out, obj)
        return out

    def barrier(self):
        if self.ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def close(self):
        if self.ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 10 ms while a timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None
        self.first = 0

    def __enter__(self):
        """Starts sampling and waits for the first sample: nvidia-smi's start-up can hold the driver
        for a moment, which must not fall inside the timed region."""
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "10"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 20 and os.path.getsize(self.path) == 0:
            time.sleep(0.05)
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
            self.proc = None

    def summary(self):
        self.__exit__(None, None, None)
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
        self.path = None
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


def source_stamp() -> str:
    """Digest of the CUDA sources, the C header and the build flags: a profile summary captured from
    another build does not describe the library being timed."""
    from mobileraytracer_b200 import build as b
    h = hashlib.sha256()
    files = sorted(f for f in os.listdir(b.CSRC) if f.endswith((".cu", ".cuh", ".h")))
    for f in files:
        h.update(f.encode())
        h.update(open(os.path.join(b.CSRC, f), "rb").read())
    h.update(open(os.path.join(ROOT, "include", "mrt_cuda.h"), "rb").read())
    h.update(" ".join(b.NVCC_FLAGS).encode())
    return h.hexdigest()[:16]


def profile_figures(path: str) -> dict:
    """`key: value` lines of a committed ncu summary (figures per launch of its kernel)."""
    out = {}
    if not os.path.exists(path):
        return out
    for line in open(path):
        line = line.strip()
        if ":" in line and not line.startswith(("|", "#", "`")) and " " not in line.split(":", 1)[0]:
            k, v = line.split(":", 1)
            v = v.strip().split()[0] if v.strip() else ""
            try:
                out[k] = float(v)
            except ValueError:
                out[k] = v
    return out


def make_soup():
    from mobileraytracer_b200 import scenes
    t0 = time.time()
    sc = scenes.triangle_soup(N_TRI, SEED, WIDTH, HEIGHT)
    log(f"scene generated in {time.time() - t0:.1f}s")
    return sc


# ---------------------------------------------------------------------------------------------
# CPU baselines: the reference's own renderer (oracle/_ref, compiled from the reference sources with
# its release optimisation level) on the host cores, on a bounded sample of the same frame
# ---------------------------------------------------------------------------------------------
def cpu_frame_baseline(sc, opts, accel: int, budget_s: float, threads: int, first: int = 0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc as O
    try:
        O.ref(fast=True)
    except Exception as e:  # the checker library was not built
        log(f"cpu baseline unavailable: {e}")
        return None
    total = WIDTH * HEIGHT
    probe_step = max(1, total // (threads * 4))
    _, n, tb, tr = O.ref_render_subset(sc, sc.camera, opts, accel, threads, first, probe_step, fast=True)
    rate = n / max(tr, 1e-6)
    step = max(1, int(total / max(1.0, rate * budget_s)))
    _, n, _, tr = O.ref_render_subset(sc, sc.camera, opts, accel, threads, first + 1, step, fast=True)
    name = {1: "RegularGrid (G by the reference rule)", 2: "BVH"}.get(accel, str(accel))
    return {"value": n / tr / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "sample": f"every {step}th pixel of the {WIDTH}x{HEIGHT} frame ({n} camera rays), reference {name} "
                      f"(build {tb:.2f}s), {threads} threads", "rays": n, "seconds": tr, "build_seconds": tb}


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


def run_reference(args):
    """--impl reference: the reference's own CPU implementation of the path on the host cores."""
    ws, rank, local = dist_info()
    if rank != 0:
        return
    from mobileraytracer_b200 import capi
    sc = make_soup()
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
        "config": {"workload": REF_WORKLOAD, "sample_per_step": f"every {step}th pixel", "accelerator": "reference BVH"},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "reference",
                         "sample": f"every {step}th pixel of the {WIDTH}x{HEIGHT} frame per step, reference BVH "
                                   f"(build {tb:.2f}s), {threads} threads"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# frames
# ---------------------------------------------------------------------------------------------
def time_frames(dist, ctx, scene, sc, opts, steps: int, warmup: int, accum: bool = False):
    """Device time of `steps` renders on device buffers, L2 flushed (512 MiB write outside the timed
    events) before every frame; clocks sampled during the timed frames.  Returns the summed frame
    time, rays, paths, the clock record, the summed time of the traversal launches and the count of
    the library's kernel launches (MrtRenderStats.kernel_launches)."""
    import torch
    w, h = opts.width, opts.height
    bitmap = torch.zeros(w * h, dtype=torch.int32, device=dist.device)
    acc = torch.zeros((h, w, 4), dtype=torch.float32, device=dist.device) if accum else None
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=dist.device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dist.device)

    def step():
        with torch.cuda.stream(stream):
            flush.fill_(1)
        return scene.render(sc.camera, opts, bitmap=bitmap, accum=acc)[2]

    clocks = ClockSampler(dist.local).__enter__()
    for _ in range(warmup):
        step()
    dist.barrier()
    torch.cuda.synchronize()
    clocks.mark()
    dev_ms, trace_ms, rays, paths, launches = 0.0, 0.0, 0, 0, 0
    for _ in range(steps):
        st = step()
        dev_ms += st.device_ms
        trace_ms += st.trace_ms
        launches += st.kernel_launches
        rays += st.rays_closest + st.rays_shadow
        paths += st.paths
    torch.cuda.synchronize()
    clk = clocks.summary()
    del flush
    return dev_ms, rays, paths, clk, trace_ms, launches


def time_e2e(scene, sc, opts, n: int, accum: bool = False):
    """End to end through the C ABI with host buffers (pinned): bitmap (and sums) in, render, out."""
    import torch
    w, h = opts.width, opts.height
    host_bm = torch.zeros((h, w), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    host_acc = torch.zeros((h, w, 4), dtype=torch.float32).pin_memory().numpy() if accum else None
    scene.render(sc.camera, opts, bitmap=host_bm, accum=host_acc)
    t = time.perf_counter()
    for _ in range(n):
        scene.render(sc.camera, opts, bitmap=host_bm, accum=host_acc)
    e2e_s = (time.perf_counter() - t) / n
    # the block schedule of these frames is the plain rectangle of rows 0 .. 16 * (h // 16) - 1, and
    # only those rows travel: in, the sums (a first pass overwrites the bitmap rows without reading
    # them), the camera and the options; out, the bitmap rows (and sums)
    rows_px = w * 16 * (h // 16)
    acc_bytes = 16 * rows_px if accum else 0
    return e2e_s, acc_bytes + 64 + 100, 4 * rows_px + acc_bytes


def soup_frame(dist, ctx, sc, args, accel: int, mode: int, grid_size: int = 0, grid_index: int = 0,
               with_cpu: bool = True, profile: str | None = None):
    """The 1920x1080 NoShadows frame of the soup on one accelerator: Mrays/s, e2e, roofline with the
    algorithmic bytes of a counting replay of the same traversal over the same camera rays."""
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import camera as mcam
    from mobileraytracer_b200 import capi
    t0 = time.time()
    scene = m.Scene(ctx, sc).build(accel, mode, grid_size=grid_size, grid_index=grid_index)
    build_s = time.time() - t0
    info = scene.accel_info()
    opts = capi.render_opts(shader=capi.MRT_SHADER_NOSHADOWS, width=WIDTH, height=HEIGHT, spp=1, spl=1)
    dev_ms, rays, _, clk, trace_ms, launches = time_frames(dist, ctx, scene, sc, opts, args.steps, args.warmup)
    dev_ms = dist.max(dev_ms)
    trace_ms = dist.max(trace_ms) / args.steps   # the traversal launch of each frame (FAST BVH)
    rays_per_step = rays // args.steps
    value = rays_per_step * args.steps * dist.ws / (dev_ms / 1e3) / 1e6
    ms = dev_ms / args.steps
    e2e_s, h2d, d2h = time_e2e(scene, sc, opts, max(1, min(args.e2e_steps, args.steps)))
    e2e_s = dist.max(e2e_s)
    rays_np = mcam.primary_rays(sc.camera, WIDTH, HEIGHT, pixels=np.arange(WIDTH * 16 * (HEIGHT // 16)))
    nodes, tris = scene.trace_counts(rays_np)
    hits = scene.trace_closest(rays_np)
    n_hit = int(np.sum((hits["id"] >> 30) == capi.MRT_PRIM_TRIANGLE))
    peak, peak_kind = measured_peak()
    n_nodes, n_tris = int(nodes.sum(dtype=np.int64)), int(tris.sum(dtype=np.int64))
    shade = {"name": "k_ns_shade (per pixel: hit record 8 + triangle record 48 + shading 76 per hit + bitmap 8)",
             "algorithmic_bytes_per_launch": 16 * len(rays_np) + (48 + 76) * n_hit, "ms": ms - trace_ms}
    if accel == capi.MRT_ACCEL_REGULAR_GRID:
        # the traversal kernel: cells 8 (start[c], start[c + 1]) + per reference 4 (index) + 48 (A, AB, AC)
        # + the 8-byte hit record written
        alg = 8 * len(rays_np) + 8 * n_nodes + 52 * n_tris
        counts = {"cells_per_ray": n_nodes / len(rays_np), "refs_per_ray": n_tris / len(rays_np),
                  "kernel_ms": trace_ms, "frame_ms": ms, "shade_kernel": shade}
        kernel = "k_ns_trace_grid (persistent grid walk; k_ns_shade shades the frame's samples after it)"
    else:
        # the traversal kernel: node bytes + 48 per triangle record + the 8-byte hit record written
        alg = FAST_NODE_BYTES * n_nodes + 48 * n_tris + 8 * len(rays_np)
        counts = {"node_fetches_per_ray": n_nodes / len(rays_np), "node_fetch_bytes": FAST_NODE_BYTES,
                  "tri_records_per_ray": n_tris / len(rays_np), "kernel_ms": trace_ms, "frame_ms": ms,
                  "shade_kernel": shade}
        kernel = "k_ns_trace (persistent traversal; k_ns_shade shades the frame's samples after it)"
    kernel_ms = trace_ms if trace_ms > 0 else ms
    achieved = alg / (kernel_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "note": ("algorithmic bytes are the node, triangle and hit records the traversal fetches; the scene "
                     "stays in L2, so they are served by L1/L2 and frac can exceed 1; dram_frac (from the ncu "
                     "capture of this source) is the DRAM use"),
            "peak_source": peak_kind, "traffic": None, "algorithmic_bytes_per_launch": alg,
            "bytes_per_ray": alg / len(rays_np), **counts, "kernel": kernel}
    if profile:
        prof = profile_figures(profile)
        stamp = source_stamp()
        if prof.get("source_sha16") == stamp and prof.get("dram_bytes_per_launch"):
            scale = len(rays_np) / float(prof.get("rays_per_launch", len(rays_np)))
            traffic = float(prof["dram_bytes_per_launch"]) * scale
            roof["traffic"] = traffic
            roof["dram_frac"] = traffic / (kernel_ms / 1e3) / 1e9 / peak
            for k in ("l1_hit_pct", "l2_hit_pct", "l1_throughput_pct", "l2_throughput_pct", "dram_throughput_pct",
                      "alu_pipe_pct", "fma_pipe_pct", "warps_active_pct", "lanes_active_per_inst", "issue_active_pct"):
                if k in prof:
                    roof[k] = prof[k]
            # the unit that actually limits the kernel: the busiest of the ones ncu measured
            units = {"L1 throughput": prof.get("l1_throughput_pct"), "ALU pipe": prof.get("alu_pipe_pct"),
                     "L2 throughput": prof.get("l2_throughput_pct"), "DRAM throughput": prof.get("dram_throughput_pct")}
            units = {k: v for k, v in units.items() if isinstance(v, float)}
            if units:
                top = max(units, key=units.get)
                roof["limiter"] = f"{top} {units[top]:.0f} % of peak (ncu); DRAM {units.get('DRAM throughput', 0):.1f} %"
            roof["profile"] = os.path.relpath(profile, ROOT) + f" (ncu capture of this source, {stamp})"
        else:
            roof["profile"] = (os.path.relpath(profile, ROOT) + " describes another build of the kernel "
                               f"(source {prof.get('source_sha16')} vs {stamp}): traffic not reported")
    cpu = None
    if with_cpu and dist.rank == 0 and dist.ws == 1 and not args.no_cpu_baseline:
        ref_accel = capi.MRT_ACCEL_REGULAR_GRID if accel == capi.MRT_ACCEL_REGULAR_GRID else capi.MRT_ACCEL_BVH
        cpu = cpu_frame_baseline(sc, opts, ref_accel, args.cpu_budget, os.cpu_count() or 1)
    rec = {"value": value, "unit": "Mrays/s", "ms_per_step": ms, "rays_per_step": rays_per_step,
           "build_seconds": build_s, "accel_info": info,
           "e2e": {"value": rays_per_step * dist.ws / e2e_s / 1e6, "unit": "Mrays/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "gpu_launches": launches, "roofline": roof, "clocks": clk, "cpu_baseline": cpu}
    scene.close()
    return rec


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


def scene_frame(dist, ctx, name: str, steps: int, warmup: int, args):
    """Configs 1 and 3: one step = one Renderer::renderFrame of the frame (mrt_render on device
    buffers); value = rays traced (camera + secondary + shadow) / device time."""
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import capi
    sc, opts = scene_workload(name)
    t0 = time.time()
    scene = m.Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    build_s = time.time() - t0
    dev_ms, rays, paths, clk, _, launches = time_frames(dist, ctx, scene, sc, opts, steps, warmup, accum=True)
    dev_ms = dist.max(dev_ms)
    value = rays * dist.ws / (dev_ms / 1e3) / 1e6
    rays_per_path = rays / paths
    e2e_s, h2d, d2h = time_e2e(scene, sc, opts, max(1, min(args.e2e_steps, steps)), accum=True)
    e2e_s = dist.max(e2e_s)
    cpu = None
    if dist.rank == 0 and dist.ws == 1 and not args.no_cpu_baseline:
        cpu = scene_cpu_baseline(sc, opts, rays_per_path, args.cpu_budget)
    scene.close()
    return {"workload": SCENE_WORKLOADS[name], "value": value, "unit": "Mrays/s", "ms_per_step": dev_ms / steps,
            "steps": steps, "rays_per_step": rays / steps, "paths_per_step": paths / steps,
            "rays_per_path": rays_per_path, "samples_per_s": paths * dist.ws / (dev_ms / 1e3),
            "bvh_build_seconds": build_s,
            "e2e": {"value": rays / steps * dist.ws / e2e_s / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches, "clocks": clk, "cpu_baseline": cpu}


# ---------------------------------------------------------------------------------------------
# batched and served
# ---------------------------------------------------------------------------------------------
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
    if not jobs:
        return []
    with mp.get_context("spawn").Pool(max(1, min(workers, len(jobs)))) as pool:
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


def batched_vs_plain(dist, args, host=None, jobs=None):
    """The 256-job batch: the batched renderer against the plain one-job-per-launch renderer on the
    same job list.  One step = every job rendered once; value = rays traced / wall time of the step
    (the batch's work spans many launches on several streams, so the step is timed on the host with
    the device synchronised on both sides).  Under torchrun the jobs are split across ranks by cost."""
    from mobileraytracer_b200 import distributed, scenes
    all_jobs = scenes.batched_jobs(args.jobs)
    if jobs is None:
        jobs = distributed.shard_jobs(all_jobs, dist.ws, dist.rank)
        host = generate_jobs(jobs, min(16, os.cpu_count() or 1))
    import torch
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import capi
    ctx = m.Context(dist.local)
    t0 = time.time()
    built = [m.Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST) for sc in host]
    build_s = time.time() - t0
    arena_bytes = sum(b.device_bytes() for b in built)
    opts = [job_opts(j, capi) for j in jobs]
    bm_plain = [torch.zeros(j.side * j.side, dtype=torch.int32, device=dist.device) for j in jobs]
    bm_batch = [torch.zeros(j.side * j.side, dtype=torch.int32, device=dist.device) for j in jobs]
    paths = sum(j.side * j.side * j.spp for j in jobs)
    per_job = {}

    def plain_step():
        rays = 0
        torch.cuda.synchronize()
        t = time.perf_counter()
        for k in range(len(jobs)):
            _, _, st = built[k].render(host[k].camera, opts[k], bitmap=bm_plain[k])
            rays += st.rays_closest + st.rays_shadow
            per_job[k] = (st.rays_closest + st.rays_shadow, st.device_ms)
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
        for k in range(len(jobs)):
            batch.submit(built[k], host[k].camera, opts[k], bm_batch[k])
        batch.run()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        batch.completed()
        s1 = batch.stats()
        return (s1.rays_closest + s1.rays_shadow) - (s0.rays_closest + s0.rays_shadow), dt, s1.busy_ms - s0.busy_ms

    steps = args.batch_steps
    clocks = ClockSampler(dist.local).__enter__()
    for _ in range(args.warmup):
        batch_step()
    plain_step()
    dist.barrier()
    clocks.mark()
    b_rays = b_time = b_busy = 0.0
    for _ in range(steps):
        r, dt, busy = batch_step()
        b_rays += r
        b_time += dt
        b_busy += busy
    p_rays = p_time = 0.0
    for _ in range(steps):
        r, dt = plain_step()
        p_rays += r
        p_time += dt
    clk = clocks.summary()
    same = sum(int(torch.equal(a, b)) for a, b in zip(bm_plain, bm_batch))
    st = batch.stats()
    b_rays, p_rays, same = dist.sum(b_rays), dist.sum(p_rays), int(dist.sum(same))
    b_time, p_time = dist.max(b_time), dist.max(p_time)
    value = b_rays / b_time / 1e6
    plain_value = p_rays / p_time / 1e6
    # what batching can gain at most: every ray at the rate of the fastest job the plain renderer ran
    # alone (jobs of at least 2^24 rays, where launch and tail costs are amortised)
    rates = [r / ms / 1e3 for r, ms in per_job.values() if r >= (1 << 24) and ms > 0]
    best = dist.max(max(rates) if rates else 0.0)   # every rank takes part in the collective
    # the plain renderer's time on small jobs (launch- and tail-bound, where batching gains) against its
    # aggregate rate on the large ones (where it already runs as a full-device persistent launch)
    big = [(r, ms) for r, ms in per_job.values() if r >= (1 << 24)]
    small = [(r, ms) for r, ms in per_job.values() if r < (1 << 24)]
    big_rays, big_ms = dist.sum(sum(r for r, _ in big)), dist.sum(sum(ms for _, ms in big))
    small_rays, small_ms = dist.sum(sum(r for r, _ in small)), dist.sum(sum(ms for _, ms in small))
    big_rate = big_rays / big_ms / 1e3 if big_ms > 0 else 0.0
    rec = {"workload": BATCH_WORKLOAD, "value": value, "unit": "Mrays/s", "ms_per_step": b_time * 1e3 / steps,
           "steps": steps, "jobs": len(all_jobs), "paths_per_step": dist.sum(paths),
           "triangles": sum(j.n_triangles for j in all_jobs), "scene_device_bytes": dist.sum(arena_bytes),
           "scene_build_seconds": build_s, "rays_per_step": b_rays / steps,
           "l2": "inputs (scenes of several GB) far larger than L2",
           "policy": args.policy, "wave_roots": st.wave_roots, "block_threads": st.block_threads,
           "blocks_per_sm": st.blocks_per_sm, "pipelines": st.pipelines, "autotuner_probes": st.autotuned,
           "whole_path_waves": st.waves_paths, "waves_per_step": st.waves / (args.warmup + steps),
           "device_busy_fraction": b_busy / 1e3 / max(b_time, 1e-9),
           "plain": {"value": plain_value, "unit": "Mrays/s", "ms_per_step": p_time * 1e3 / steps,
                     "rays_per_step": p_rays / steps, "renderer": "mrt_render per job, device buffers"},
           "batched_over_plain": value / plain_value, "bitmaps_equal_plain": f"{same}/{len(all_jobs)}",
           "plain_best_job_Mrays_per_s": best,
           "ratio_bound_at_best_job_rate": (best / plain_value) if best else None,
           "plain_large_jobs": {"jobs": int(dist.sum(len(big))), "rays": big_rays, "device_ms": big_ms,
                                "Mrays_per_s": big_rate, "rule": "jobs of at least 2^24 rays"},
           "plain_small_jobs": {"jobs": int(dist.sum(len(small))), "rays": small_rays, "device_ms": small_ms,
                                "Mrays_per_s": small_rays / small_ms / 1e3 if small_ms > 0 else None},
           "ratio_bound_at_large_job_rate": (big_rate / plain_value) if big_rate else None,
           "clocks": clk}
    batch.close()
    for b in built:
        b.close()
    ctx.close()
    return rec


SERVE_WORKLOAD = ("Poisson stream of render requests, each drawn as a batched-workload job (PathTracer "
                  "depth 6, soup geometry from the 256-job pool, side log-uniform over [128, 1024], spp uniform "
                  "over {1, 4, 16, 64}); 20% re-render one of the last 64 new scenes with +16 spp progressive "
                  "accumulation; admission by device footprint")


def served_vs_plain(dist, args, duration: float, rate: float, host=None):
    """The request stream served by the batched renderer (continuous batching) and by one mrt_render
    call per request: throughput, p50/p99 latency (arrival to result), offered vs achieved load, and
    whether every result equals the one-render-per-request result.  Under torchrun every rank serves
    the requests of the scenes whose id is its rank modulo the world size (a progressive re-render goes
    to the rank that holds its scene), at their own arrival times."""
    from mobileraytracer_b200 import scenes
    from mobileraytracer_b200 import serve
    pool = scenes.batched_jobs(256)
    if host is None:
        host = generate_jobs(pool, min(16, os.cpu_count() or 1))
    all_reqs = serve.request_stream(pool, duration_s=duration, rate=rate)
    reqs = [r for r in all_reqs if r.scene % dist.ws == dist.rank] if dist.ws > 1 else all_reqs
    if dist.ws > 1:   # the loop indexes its requests 0..n-1 and re-renders refer to a scene's first request
        import dataclasses
        remap = {r.index: k for k, r in enumerate(reqs)}
        reqs = [dataclasses.replace(r, index=remap[r.index], scene=remap[r.scene]) for r in reqs]
    offered_paths = sum(r.paths for r in all_reqs)
    import torch
    import mobileraytracer_b200 as m
    budget = int(args.budget_gb * 1e9)
    bitmap_reserve = 8 << 30          # images of every scene served (kept for progressive re-renders)
    build_slack = 1 << 30             # tree-build scratch of the scene being built
    scene_budget = budget - bitmap_reserve - build_slack

    def pool_scene(r):
        return host[r.geometry]

    results = {}
    clocks = ClockSampler(dist.local).__enter__()
    clocks.mark()
    for kind in ("plain", "batched"):
        dist.barrier()
        ctx = m.Context(dist.local)
        arena = m.Arena(dist.local, scene_budget + build_slack)
        if kind == "batched":
            be = serve.BatchBackend(ctx, arena, pool_scene, dict(
                max_depth=6, max_spl=1, max_jobs=4096, wave_roots=args.wave_roots or (1 << 20),
                max_wave_roots=max(args.wave_roots, 1 << 20), block_threads=64, blocks_per_sm=16,
                pipelines=args.pipelines or 4), device=dist.local)
        else:
            be = serve.PlainBackend(ctx, arena, pool_scene, device=dist.local)
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
        log(f"{kind} @ {rate}/s: {summary['wall_seconds']:.1f}s, p50 {summary['latency_p50_s']:.3f}s p99 "
            f"{summary['latency_p99_s']:.3f}s, {summary['rays'] / summary['wall_seconds'] / 1e6:.1f} Mrays/s")
    clk = clocks.summary()
    same = sum(int(results["plain"]["checksums"][i] == results["batched"]["checksums"][i]) for i in range(len(reqs)))

    def summ(r):
        rec = r["records"]
        lat = np.concatenate(dist.gather(np.array([rec[i]["done"] - rec[i]["arrival"] for i in range(len(reqs))])))
        wall = dist.max(r["wall_seconds"])
        rays = dist.sum(r["rays"])
        p99 = float(np.percentile(lat, 99)) if len(lat) else 0.0
        return {"Mrays_per_s": rays / wall / 1e6, "wall_seconds": wall,
                "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else 0.0, "latency_p99_s": p99,
                "latency_mean_s": float(lat.mean()) if len(lat) else 0.0, "achieved_paths_per_s": offered_paths / wall,
                # the backlog does not grow: the run ends within 5 % of the arrival window plus one
                # second to drain the requests that arrived last
                "keeps_up": bool(wall <= duration * 1.05 + 1.0),
                "rays": rays, "evictions": int(dist.sum(r["evictions"])),
                "rebuilds_after_eviction": int(dist.sum(r["rebuilds_after_eviction"])),
                "peak_scene_bytes": dist.max(r["peak_scene_bytes"]), "arena_peak_bytes": dist.max(r["arena"]["peak"])}

    p = summ(results["plain"])
    b = summ(results["batched"])
    same = int(dist.sum(same))
    return {"workload": SERVE_WORKLOAD, "duration_s": duration, "rate_per_s": rate, "requests": len(all_reqs),
            "rerenders": sum(r.kind == "rerender" for r in all_reqs),
            "offered_paths_per_s": offered_paths / duration, "budget_bytes": budget, "scene_budget_bytes": scene_budget,
            "served": b, "plain": p, "served_over_plain": b["Mrays_per_s"] / p["Mrays_per_s"],
            "results_equal_plain": f"{same}/{len(all_reqs)}", "clocks": clk}


# ---------------------------------------------------------------------------------------------
# raster preview
# ---------------------------------------------------------------------------------------------
def raster_line(dist, args):
    """The raster preview of the 1920x1080 frame's soup (1,000,000 triangles, 1920x1080): one step = one
    mrt_raster_preview on a device bitmap; value = scene triangles / device time (Mtris/s)."""
    import torch
    import mobileraytracer_b200 as m
    w, h = WIDTH, HEIGHT
    sc = make_soup()
    ctx = m.Context(dist.local)
    scene = m.Scene(ctx, sc)
    bitmap = torch.zeros((h, w), dtype=torch.int32, device=dist.device)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=dist.device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dist.device)

    def step():
        with torch.cuda.stream(stream):
            flush.fill_(1)   # evicts L2 before every step; not inside the timed events
        return scene.raster_preview(sc.camera, w, h, bitmap=bitmap)[1]

    clocks = ClockSampler(dist.local).__enter__()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks.mark()
    dev_ms, st = 0.0, None
    for _ in range(args.steps):
        st = step()
        dev_ms += st.device_ms
    torch.cuda.synchronize()
    clk = clocks.summary()
    ms = dist.max(dev_ms) / args.steps
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
    e2e_s = dist.max((time.perf_counter() - t1) / n_e2e)
    cpu = None
    if not args.no_cpu_baseline and dist.rank == 0 and dist.ws == 1:
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
        "metric": METRIC, "value": sc.n_triangles * dist.ws / (ms / 1e3) / 1e6, "unit": "Mtris/s",
        "n_gpus": dist.ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "raster preview (MainRenderer.copyFrame) of the 1,000,000-triangle soup seed 0, "
                               "1920x1080, the CLI camera", "triangles": sc.n_triangles, "drawn": st.drawn,
                   "fragments": st.fragments, "covered_pixels": covered,
                   "l2": "flushed before every step (512 MiB write outside the timed events)"},
        "e2e": {"value": sc.n_triangles * dist.ws / e2e_s / 1e6, "unit": "Mtris/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": host_bm.nbytes},
        "gpu_launches": 3 * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": None, "algorithmic_bytes_per_launch": algo,
                     "kernel": "k_raster_tris + k_raster_big + k_raster_resolve (+ key clear)"},
        "clocks": clk, "cpu_baseline": cpu,
    }
    scene.close()
    ctx.close()
    return line


# ---------------------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20, help="timed frames of each frame workload")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--cpu-budget", type=float, default=10.0, help="seconds of reference CPU work per cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="all",
                    choices=["all", "frame", "grid", "cornell", "terrain", "batched", "served", "served-sweep", "raster"],
                    help="all: the headline frame and every other configuration in one line (default); frame: "
                         "the headline frame alone; grid: the frame on the RegularGrid; cornell / terrain: the "
                         "Whitted and PathTracer frames; batched: the 256-job batch; served: the request stream; "
                         "served-sweep: the stream at rising arrival rates; raster: the raster preview")
    ap.add_argument("--terrain-steps", type=int, default=3)
    ap.add_argument("--batch-steps", type=int, default=1)
    ap.add_argument("--duration", type=float, default=None, help="served: seconds of arrivals (default 30; 120 alone)")
    ap.add_argument("--rate", type=float, default=50.0, help="served: arrivals per second")
    ap.add_argument("--rates", default="50,100,200,400", help="served-sweep: arrival rates")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="served: device footprint budget")
    ap.add_argument("--pipelines", type=int, default=0, help="batched/served: waves in flight (0: autotuned / 4)")
    ap.add_argument("--jobs", type=int, default=256, help="batched: jobs in the list")
    ap.add_argument("--wave-roots", type=int, default=0, help="batched: camera paths per wave (0: autotuned)")
    ap.add_argument("--policy", default="smallest", choices=["smallest", "fifo", "share"],
                    help="batched: which jobs fill a wave")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args)
        return

    dist = Dist()
    import mobileraytracer_b200 as m
    from mobileraytracer_b200 import capi

    def emit(line):
        if dist.rank == 0:
            print(json.dumps(line), flush=True)

    base = {"metric": METRIC, "n_gpus": dist.ws, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    if args.workload == "raster":
        emit(raster_line(dist, args))
        dist.close()
        return
    if args.workload in ("batched", "served", "served-sweep"):
        if args.workload == "batched":
            rec = batched_vs_plain(dist, args)
            val = rec["value"]
        elif args.workload == "served":
            rec = served_vs_plain(dist, args, args.duration or 120.0, args.rate)
            val = rec["served"]["Mrays_per_s"]
        else:
            from mobileraytracer_b200 import scenes
            host = generate_jobs(scenes.batched_jobs(256), min(16, os.cpu_count() or 1))
            sweep = [served_vs_plain(dist, args, args.duration or 30.0, float(r), host=host)
                     for r in args.rates.split(",")]
            rec = {"workload": SERVE_WORKLOAD, "sweep": sweep}
            for kind in ("served", "plain"):   # capacity: the most rays per second either server sustained
                kept = [s["rate_per_s"] for s in sweep if s[kind]["keeps_up"]]
                rec[f"{kind}_capacity"] = {"Mrays_per_s": max(s[kind]["Mrays_per_s"] for s in sweep),
                                          "highest_rate_kept_up": max(kept) if kept else None}
            rec["capacity_ratio"] = rec["served_capacity"]["Mrays_per_s"] / rec["plain_capacity"]["Mrays_per_s"]
            val = rec["served_capacity"]["Mrays_per_s"]
        emit({**base, "value": val, "unit": "Mrays/s", "steps": 1, "ms_per_step": rec.get("ms_per_step"),
              "config": {"workload": rec["workload"]}, args.workload: rec})
        dist.close()
        return
    if args.workload in SCENE_WORKLOADS:
        steps = args.terrain_steps if args.workload == "terrain" else args.steps
        ctx = m.Context(dist.local)
        rec = scene_frame(dist, ctx, args.workload, steps, args.warmup, args)
        ctx.close()
        emit({**base, "value": rec["value"], "unit": "Mrays/s", "steps": steps, "ms_per_step": rec["ms_per_step"],
              "config": {"workload": rec["workload"], "l2": "flushed before every step (512 MiB write outside the "
                                                             "timed events)"},
              "e2e": rec["e2e"], "gpu_launches": rec["gpu_launches"], "roofline": None, "clocks": rec["clocks"],
              "cpu_baseline": rec["cpu_baseline"], args.workload: rec})
        dist.close()
        return

    sc = make_soup()
    ctx = m.Context(dist.local)
    if args.workload == "grid":
        rec = soup_frame(dist, ctx, sc, args, capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST, profile=GRID_PROFILE)
        emit({**base, "value": rec["value"], "unit": "Mrays/s", "ms_per_step": rec["ms_per_step"],
              "config": {"workload": FRAME + ", RegularGrid G = 128 (the reference's sizing rule)"},
              **{k: rec[k] for k in ("e2e", "gpu_launches", "roofline", "clocks", "cpu_baseline")}})
        ctx.close()
        dist.close()
        return
    head = soup_frame(dist, ctx, sc, args, capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, profile=PROFILE)
    line = {**base, "value": head["value"], "unit": "Mrays/s", "ms_per_step": head["ms_per_step"],
            "config": {"workload": WORKLOAD, "rays_per_step": head["rays_per_step"],
                       "rows_rendered": 16 * (HEIGHT // 16),
                       "l2": "flushed before every step (512 MiB write outside the timed events)",
                       "bvh_build_seconds": head["build_seconds"], "parallelism": f"replicas x{dist.ws}"},
            "e2e": head["e2e"], "gpu_launches": head["gpu_launches"], "roofline": head["roofline"],
            "clocks": head["clocks"], "cpu_baseline": head["cpu_baseline"]}
    if args.workload == "all":
        configs = {}
        t_all = time.time()
        g128 = soup_frame(dist, ctx, sc, args, capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST, profile=GRID_PROFILE)
        configs["soup_1080p_grid_G128"] = {"workload": FRAME + ", RegularGrid with G = 128 by the reference's "
                                                               "sizing rule (Shader.cpp:76-105), reference cell indexing",
                                           **g128}
        g100 = soup_frame(dist, ctx, sc, args, capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST, grid_size=100,
                          grid_index=capi.MRT_GRID_INDEX_LINEAR, with_cpu=False)
        configs["soup_1080p_grid_G100"] = {"workload": FRAME + ", RegularGrid with G = 100 = cbrt(N) and linear "
                                                               "cell indexing (the reference's shift indexing "
                                                               "is valid only for powers of two)", **g100}
        del sc
        configs["cornell_whitted_256"] = scene_frame(dist, ctx, "cornell", args.steps, args.warmup, args)
        configs["terrain_pathtracer_1024_64spp"] = scene_frame(dist, ctx, "terrain", args.terrain_steps,
                                                               args.warmup, args)
        ctx.close()
        from mobileraytracer_b200 import distributed, scenes
        jobs = distributed.shard_jobs(scenes.batched_jobs(args.jobs), dist.ws, dist.rank)
        host_jobs = generate_jobs(jobs, min(16, os.cpu_count() or 1))
        configs["batched_256_jobs"] = batched_vs_plain(dist, args, host=host_jobs, jobs=jobs)
        pool_host = host_jobs if (args.jobs == 256 and dist.ws == 1) else None   # the served pool: the same 256 jobs
        configs["served_stream"] = served_vs_plain(dist, args, args.duration or 30.0, args.rate, host=pool_host)
        line["configs"] = configs
        line["configs_seconds"] = time.time() - t_all
    else:
        ctx.close()
    emit(line)
    dist.close()


if __name__ == "__main__":
    main()
