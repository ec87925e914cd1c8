"""Serving render requests that arrive over time (continuous batching).

The reference renders one frame per Renderer::renderFrame call and keeps no state between calls
(Renderer.cpp:31-59 restarts from sample 0); a service rendering many users' scenes needs more:

  * admission by device footprint: a request whose scene is not on the device is admitted only when
    its estimated footprint (geometry + tree, carved from the device arena) fits the budget; idle
    resident scenes are evicted, least recently used first, to make room;
  * resident scenes: a scene stays on the device after its render, so a later request for it (a
    progressive re-render adding samples to its image) needs no upload or build; its bitmap (the
    running mean) stays as well, and the re-render continues the sample stream at spp_offset;
  * one render at a time per scene (a progressive re-render waits for the previous one), any number
    of scenes at once;
  * continuous batching: requests are handed to the batched renderer as soon as their scene is built,
    and their rays join the next waves beside the rays of requests already running.

`ServeLoop` is the policy; a backend does the device work.  `BatchBackend` submits to the batched
renderer (mrt_batch_*), `PlainBackend` renders each request with one mrt_render call (the
one-job-per-launch baseline); both build scenes on a second thread with their own context, so uploads
and tree builds overlap rendering.  The loop itself has no device code and is tested with a fake
backend.
"""
from __future__ import annotations

import collections
import heapq
import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import capi, scenes


@dataclass
class Request:
    index: int
    arrival: float        # seconds after the start of the stream
    scene: int            # scene id: index of the request that created the scene
    kind: str             # "new" or "rerender"
    geometry: int         # index of the scene's geometry in the pool
    n_triangles: int
    side: int
    spp: int
    spp_offset: int       # samples the scene's image already holds
    seed: int             # sample-stream seed of the scene

    @property
    def paths(self) -> int:
        return self.side * self.side * self.spp


def request_stream(pool: list, duration_s: float = 120.0, rate: float = 50.0, rerender_frac: float = 0.2,
                   recent: int = 64, rerender_spp: int = 16, seed: int = 2024, side_range=(128, 1024),
                   spps=(1, 4, 16, 64)) -> list[Request]:
    """Poisson arrivals at `rate` per second for `duration_s`.  A new request draws its geometry from
    `pool` (scenes.Job entries) and its image side and spp from the batched workload's distributions
    (side log-uniform over [128, 1024] in multiples of 16, spp uniform over {1, 4, 16, 64}); with
    probability `rerender_frac` a request instead re-renders one of the last `recent` new scenes with
    `rerender_spp` more samples, continuing its image."""
    out: list[Request] = []
    t = 0.0
    k = 0
    spp_of: dict[int, int] = {}
    new_ids: list[int] = []
    while True:
        u = scenes.uniform(seed * 7919 + k, 6, stream=23)
        t += -math.log1p(-u[0]) / rate
        if t > duration_s:
            break
        if new_ids and u[1] < rerender_frac:
            sid = new_ids[max(0, len(new_ids) - recent) + int(u[2] * min(recent, len(new_ids)))]
            base = out[sid]
            out.append(Request(k, t, sid, "rerender", base.geometry, base.n_triangles, base.side, rerender_spp,
                               spp_of[sid], base.seed))
            spp_of[sid] += rerender_spp
        else:
            g = int(u[3] * len(pool))
            lo, hi = side_range
            side = int(math.exp(math.log(lo) + u[4] * (math.log(hi) - math.log(lo))))
            side = max(lo, side - side % 16)
            spp = spps[min(len(spps) - 1, int(u[5] * len(spps)))]
            out.append(Request(k, t, k, "new", g, pool[g].n_triangles, side, spp, 0, 1_000_000 + k))
            spp_of[k] = spp
            new_ids.append(k)
        k += 1
    return out


def request_opts(r: Request) -> capi.MrtRenderOpts:
    """PathTracer, depth 6 with Russian roulette beyond depth 3, one light sample (the batched
    workload's settings); the reference CLI's sampler wiring for the request's spp."""
    return capi.render_opts(shader=capi.MRT_SHADER_PATHTRACER, width=r.side, height=r.side, spp=r.spp, spl=1,
                            depth_min=3, depth_max=6, seed=r.seed, spp_offset=r.spp_offset)


def scene_bytes_estimate(n_triangles: int) -> int:
    """Device bytes of a triangle-soup scene with its FAST tree (geometry 48 + shading 76 + leaf-order
    triangles 48 + about 64 of tree records per triangle, plus block rounding)."""
    return 240 * n_triangles + (1 << 20)


@dataclass
class _SceneState:
    resident: bool = False
    built: bool = False
    building: bool = False
    busy: bool = False            # a request of this scene is queued for or in rendering
    nbytes: int = 0
    waiting: collections.deque = field(default_factory=collections.deque)


class ServeLoop:
    """Admission, residency and dispatch of a request stream over a backend.

    Backend interface:
      start_build(req)            build req's scene (asynchronously)
      poll_builds() -> [(scene, nbytes or None)]   finished builds (None: no room, retry later)
      release(scene)              evict a built scene
      start_render(req)           render (batched: queue; plain: may run to completion here)
      poll_renders() -> [index]   finished requests
      can_accept() -> bool        room for another render in flight
      progress() -> bool          advance device work; True if anything was launched
      wait(seconds)               block up to `seconds` for device progress
    """

    def __init__(self, requests: list[Request], backend, scene_budget: int, clock=time.perf_counter):
        self.reqs = requests
        self.be = backend
        self.budget = scene_budget
        self.clock = clock
        self.scenes: dict[int, _SceneState] = {}
        self.idle = collections.OrderedDict()      # resident, built, idle scenes in LRU order
        self.ready: list = []                      # heap of (arrival, index)
        self.pending: collections.deque = collections.deque()
        self.used = 0
        self.peak = 0
        self.evictions = 0
        self.rebuilds = 0
        self.records: dict[int, dict] = {}

    def _available(self, sid: int):
        st = self.scenes[sid]
        if not st.built or st.busy:
            return
        if st.waiting:
            r = st.waiting.popleft()
            st.busy = True
            self.idle.pop(sid, None)
            heapq.heappush(self.ready, (r.arrival, r.index))
        else:
            self.idle[sid] = True
            self.idle.move_to_end(sid)

    def _evict_one(self) -> bool:
        if not self.idle:
            return False
        sid, _ = self.idle.popitem(last=False)
        st = self.scenes[sid]
        self.be.release(sid)
        self.used -= st.nbytes
        st.resident = st.built = False
        st.nbytes = 0
        self.evictions += 1
        return True

    def _admit(self, now: float) -> bool:
        moved = False
        while self.pending:
            r = self.pending[0]
            st = self.scenes.setdefault(r.scene, _SceneState())
            if st.resident:
                st.waiting.append(r)
                self.pending.popleft()
                self.records[r.index]["admitted"] = now
                self._available(r.scene)
                moved = True
                continue
            need = scene_bytes_estimate(r.n_triangles)
            while self.used + need > self.budget and self._evict_one():
                pass
            if self.used + need > self.budget:
                break   # the head of the queue waits for room
            self.used += need
            self.peak = max(self.peak, self.used)
            st.resident = st.building = True
            st.nbytes = need
            st.waiting.append(r)
            self.pending.popleft()
            self.records[r.index]["admitted"] = now
            if r.kind == "rerender":
                self.rebuilds += 1
            self.be.start_build(r)
            moved = True
        return moved

    def run(self) -> dict:
        n = len(self.reqs)
        nxt = 0
        done = 0
        t0 = self.clock()
        while done < n:
            now = self.clock() - t0
            active = False
            while nxt < n and self.reqs[nxt].arrival <= now:
                r = self.reqs[nxt]
                self.pending.append(r)
                self.records[r.index] = {"arrival": r.arrival, "paths": r.paths, "kind": r.kind}
                nxt += 1
                active = True
            for sid, nbytes in self.be.poll_builds():
                st = self.scenes[sid]
                st.building = False
                active = True
                if nbytes is None:           # the arena had no room: give the estimate back, retry
                    self.used -= st.nbytes
                    st.resident = False
                    st.nbytes = 0
                    while st.waiting:
                        self.pending.appendleft(st.waiting.pop())
                    self._evict_one()
                    continue
                self.used += nbytes - st.nbytes
                self.peak = max(self.peak, self.used)
                st.nbytes = nbytes
                st.built = True
                self._available(sid)
            for idx in self.be.poll_renders():
                r = self.reqs[idx]
                self.records[idx]["done"] = self.clock() - t0
                done += 1
                st = self.scenes[r.scene]
                st.busy = False
                self._available(r.scene)
                active = True
            if self._admit(self.clock() - t0):
                active = True
            while self.ready and self.be.can_accept():
                _, idx = heapq.heappop(self.ready)
                self.records[idx]["started"] = self.clock() - t0
                self.be.start_render(self.reqs[idx])
                active = True
            if self.be.progress():
                active = True
            if not active and done < n:
                wait = 0.002
                if nxt < n and not self.ready:
                    wait = min(wait, max(0.0, self.reqs[nxt].arrival - (self.clock() - t0)))
                self.be.wait(wait)
        wall = self.clock() - t0
        lat = np.array([self.records[i]["done"] - self.records[i]["arrival"] for i in range(n)])
        return {
            "requests": n, "wall_seconds": wall, "peak_scene_bytes": self.peak, "evictions": self.evictions,
            "rebuilds_after_eviction": self.rebuilds,
            "latency_p50_s": float(np.percentile(lat, 50)) if n else 0.0,
            "latency_p99_s": float(np.percentile(lat, 99)) if n else 0.0,
            "latency_mean_s": float(lat.mean()) if n else 0.0,
            "records": self.records,
        }


class _Builder:
    """Scene uploads and tree builds on a thread of their own, with a context of their own that
    shares the device arena; built scenes are handed to the rendering context."""

    def __init__(self, device: int, arena, render_ctx, pool_scene):
        import mobileraytracer_b200 as m
        self.ctx = m.Context(device)
        self.ctx.set_arena(arena)
        self.render_ctx = render_ctx
        self.pool_scene = pool_scene
        self.jobs: queue.Queue = queue.Queue()
        self.done: queue.Queue = queue.Queue()
        self.thread = threading.Thread(target=self._loop, daemon=True)
        self.thread.start()

    def _loop(self):
        import mobileraytracer_b200 as m
        while True:
            r = self.jobs.get()
            if r is None:
                return
            try:
                host = self.pool_scene(r)
                s = m.Scene(self.ctx, host).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
                s.move_to(self.render_ctx)
                self.done.put((r.scene, s))
            except m.MrtError as e:
                if e.status != capi.MRT_ERR_OOM:
                    raise
                self.done.put((r.scene, None))

    def submit(self, r: Request):
        self.jobs.put(r)

    def finished(self):
        out = []
        while True:
            try:
                out.append(self.done.get_nowait())
            except queue.Empty:
                return out

    def close(self):
        self.jobs.put(None)
        self.thread.join()
        self.ctx.close()


class _DeviceBackend:
    """What the batched and plain backends share: scenes, bitmaps, builds, result checksums."""

    def __init__(self, ctx, arena, pool_scene, device: int = 0):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.device = f"cuda:{device}"
        self.builder = _Builder(device, arena, ctx, pool_scene)
        self.scenes: dict[int, object] = {}
        self.bitmaps: dict[int, object] = {}
        self.checksums: dict[int, int] = {}
        self.weights = None
        self.rays = 0

    def start_build(self, r: Request):
        self.builder.submit(r)

    def poll_builds(self):
        out = []
        for sid, s in self.builder.finished():
            if s is None:
                out.append((sid, None))
            else:
                self.scenes[sid] = s
                out.append((sid, s.device_bytes()))
        return out

    def release(self, sid: int):
        s = self.scenes.pop(sid)
        s.close()

    def bitmap(self, r: Request):
        bm = self.bitmaps.get(r.scene)
        if bm is None:
            bm = self.torch.zeros(r.side * r.side, dtype=self.torch.int32, device=self.device)
            self.bitmaps[r.scene] = bm
        return bm

    def checksum(self, r: Request):
        torch = self.torch
        bm = self.bitmaps[r.scene]
        if self.weights is None or self.weights.numel() < bm.numel():
            g = torch.Generator(device="cpu").manual_seed(1)
            self.weights = torch.randint(1, 2 ** 31 - 1, (1 << 20,), generator=g, dtype=torch.int64).cuda()
        v = (bm.to(torch.int64) & 0xFFFFFFFF) * self.weights[:bm.numel()]
        self.checksums[r.index] = int(v.sum().item())

    def close(self):
        self.builder.close()
        for s in self.scenes.values():
            s.close()
        self.scenes.clear()


class BatchBackend(_DeviceBackend):
    """Requests join the batched renderer's waves as soon as their scene is ready."""

    def __init__(self, ctx, arena, pool_scene, batch_kwargs: dict, device: int = 0):
        super().__init__(ctx, arena, pool_scene, device)
        import mobileraytracer_b200 as m
        self.batch = m.Batch(ctx, **batch_kwargs)
        self.by_id: dict[int, Request] = {}
        self.s0 = self.batch.stats()

    def start_render(self, r: Request):
        jid = self.batch.submit(self.scenes[r.scene], self.scene_camera(r), request_opts(r), self.bitmap(r))
        self.by_id[jid] = r

    def scene_camera(self, r: Request):
        return scenes.cli_camera(r.side, r.side)

    def can_accept(self) -> bool:
        return len(self.by_id) < 4000

    def progress(self) -> bool:
        return self.batch.step(2) > 0

    def poll_renders(self):
        out = []
        for jid in self.batch.completed():
            r = self.by_id.pop(jid)
            self.checksum(r)
            out.append(r.index)
        return out

    def wait(self, seconds: float):
        time.sleep(seconds)

    def total_rays(self) -> int:
        s = self.batch.stats()
        return (s.rays_closest + s.rays_shadow) - (self.s0.rays_closest + self.s0.rays_shadow)

    def close(self):
        self.batch.run()
        self.batch.close()
        super().close()


class PlainBackend(_DeviceBackend):
    """One mrt_render call per request, in arrival order of the ready requests."""

    def __init__(self, ctx, arena, pool_scene, device: int = 0):
        super().__init__(ctx, arena, pool_scene, device)
        self.finished: list[int] = []

    def start_render(self, r: Request):
        _, _, st = self.scenes[r.scene].render(scenes.cli_camera(r.side, r.side), request_opts(r), bitmap=self.bitmap(r))
        self.rays += st.rays_closest + st.rays_shadow
        self.checksum(r)
        self.finished.append(r.index)

    def can_accept(self) -> bool:
        return not self.finished   # one render at a time; the loop collects it first

    def progress(self) -> bool:
        return False

    def poll_renders(self):
        out, self.finished = self.finished, []
        return out

    def wait(self, seconds: float):
        time.sleep(seconds)

    def total_rays(self) -> int:
        return self.rays
