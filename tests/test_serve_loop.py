"""The serving loop's policy (admission by footprint, residency, eviction, per-scene ordering of
progressive re-renders) with a fake backend on the CPU: no device involved."""
import collections

import numpy as np

from mobileraytracer_b200 import scenes, serve


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class FakeBackend:
    """Builds take `build_s`, renders `render_s` per million paths; several renders at once."""

    def __init__(self, clock, loop_ref, build_s=0.01, render_s=0.02, max_inflight=8):
        self.clock = clock
        self.loop_ref = loop_ref
        self.build_s, self.render_s, self.max_inflight = build_s, render_s, max_inflight
        self.builds = []        # (t_done, scene)
        self.renders = []       # (t_done, index)
        self.built = set()
        self.rendering = collections.Counter()
        self.order = collections.defaultdict(list)   # scene -> request indices in render order
        self.max_used = 0
        self.released = []

    def _check_budget(self):
        loop = self.loop_ref[0]
        self.max_used = max(self.max_used, loop.used)
        assert loop.used <= loop.budget

    def start_build(self, r):
        assert r.scene not in self.built
        self.builds.append((self.clock() + self.build_s, r.scene, r.n_triangles))
        self._check_budget()

    def poll_builds(self):
        now = self.clock()
        out = [(s, serve.scene_bytes_estimate(n) - 4096) for t, s, n in self.builds if t <= now]
        self.builds = [b for b in self.builds if b[0] > now]
        for s, _ in out:
            self.built.add(s)
        return out

    def release(self, sid):
        assert sid in self.built and self.rendering[sid] == 0
        self.built.discard(sid)
        self.released.append(sid)

    def start_render(self, r):
        assert r.scene in self.built, "render before the scene was built"
        assert self.rendering[r.scene] == 0, "two renders of one scene at once"
        self.rendering[r.scene] += 1
        self.order[r.scene].append(r.index)
        self.renders.append((self.clock() + self.render_s * (1 + r.paths / 1e6), r.index, r.scene))
        self._check_budget()

    def poll_renders(self):
        now = self.clock()
        out = [(i, s) for t, i, s in self.renders if t <= now]
        self.renders = [x for x in self.renders if x[0] > now]
        for _, s in out:
            self.rendering[s] -= 1
        return [i for i, _ in out]

    def can_accept(self):
        return len(self.renders) < self.max_inflight

    def progress(self):
        return False

    def wait(self, seconds):
        self.clock.t += max(seconds, 1e-4)


def run(reqs, budget, **kw):
    clock = FakeClock()
    ref = [None]
    be = FakeBackend(clock, ref, **kw)
    loop = serve.ServeLoop(reqs, be, budget, clock=clock)
    ref[0] = loop
    out = loop.run()
    return loop, be, out


def test_request_stream_shape():
    pool = scenes.batched_jobs(32)
    reqs = serve.request_stream(pool, duration_s=40.0, rate=50.0)
    assert reqs == serve.request_stream(pool, duration_s=40.0, rate=50.0)    # deterministic
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0) and arr[-1] <= 40.0
    assert abs(len(reqs) / 40.0 - 50.0) < 5.0
    frac = np.mean([r.kind == "rerender" for r in reqs])
    assert 0.15 < frac < 0.25
    spp = collections.defaultdict(int)
    for r in reqs:
        if r.kind == "new":
            assert r.scene == r.index and r.spp_offset == 0 and r.spp in (1, 4, 16, 64)
            assert 128 <= r.side <= 1024 and r.side % 16 == 0
        else:
            base = reqs[r.scene]
            assert base.kind == "new" and r.side == base.side and r.seed == base.seed and r.spp == 16
            assert r.spp_offset == spp[r.scene], "a re-render continues where the image stands"
        spp[r.scene] += r.spp


def test_every_request_served_in_order_within_budget():
    pool = scenes.batched_jobs(16)
    reqs = serve.request_stream(pool, duration_s=10.0, rate=50.0)
    budget = 12 * serve.scene_bytes_estimate(2_000_000)
    loop, be, out = run(reqs, budget)
    assert len(loop.records) == len(reqs) and all("done" in r for r in loop.records.values())
    assert be.max_used <= budget
    for sid, order in be.order.items():      # per scene: arrival order, hence spp_offset order
        assert order == sorted(order)
        offs = [reqs[i].spp_offset for i in order]
        assert offs == sorted(offs)
    lat = [loop.records[i]["done"] - loop.records[i]["arrival"] for i in range(len(reqs))]
    assert min(lat) >= 0 and out["latency_p99_s"] >= out["latency_p50_s"]


def test_small_budget_evicts_and_rebuilds():
    pool = scenes.batched_jobs(16)
    reqs = serve.request_stream(pool, duration_s=10.0, rate=50.0, recent=400)
    biggest = max(serve.scene_bytes_estimate(r.n_triangles) for r in reqs)
    loop, be, out = run(reqs, biggest + 1)   # room for about one scene at a time
    assert out["evictions"] > 0 and be.released
    assert out["rebuilds_after_eviction"] > 0   # re-renders of evicted scenes build them again
    assert be.max_used <= biggest + 1
    assert all("done" in r for r in loop.records.values())
