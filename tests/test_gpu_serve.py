"""Serving on the device (GPU): the device arena, handing scenes between contexts, and the served
stream's results, which must equal the one-request-per-launch results request by request (each
result the same alone and in the mix)."""
import numpy as np
import pytest

import mobileraytracer_b200 as m
from mobileraytracer_b200 import MrtError, capi, scenes, serve

pytestmark = pytest.mark.gpu


def test_arena_accounting(ctx):
    arena = m.Arena(0, 256 << 20)
    c2 = m.Context(0)
    c2.set_arena(arena)
    sc = scenes.triangle_soup(100000, 3, 64, 64)
    s = m.Scene(c2, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    st = arena.stats()
    assert st["used"] >= s.device_bytes() > 0 and st["peak"] >= st["used"]
    with pytest.raises(MrtError):
        arena.close()                       # a scene is still carved from it
    big = scenes.triangle_soup(1_500_000, 4, 64, 64)
    with pytest.raises(MrtError) as e:
        m.Scene(c2, big).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    assert e.value.status == capi.MRT_ERR_OOM
    # the scene renders the same after moving to another context
    o = capi.render_opts(shader=capi.MRT_SHADER_WHITTED, width=64, height=64, spp=2, seed=3)
    bm1, _, _ = s.render(sc.camera, o)
    s.move_to(ctx)
    bm2, _, _ = s.render(sc.camera, o)
    assert np.array_equal(bm1, bm2)
    s.close()
    c2.close()           # its scenes and its render scratch (also carved from the arena) go back
    assert arena.stats()["used"] == 0
    arena.close()


def _pool():
    return [scenes.Job(i, n, 128, 1, 40 + i) for i, n in enumerate((2000, 30000, 120000, 8000, 60000, 250000))]


def _serve(kind, reqs, pool, budget):
    torch = pytest.importorskip("torch")
    host = {}

    def pool_scene(r):
        if r.geometry not in host:
            host[r.geometry] = pool[r.geometry].scene()
        return host[r.geometry]

    ctx = m.Context(0)
    arena = m.Arena(0, budget + (64 << 20))
    if kind == "batched":
        be = serve.BatchBackend(ctx, arena, pool_scene, dict(max_depth=6, max_spl=1, wave_roots=20000, block_threads=128,
                                                             blocks_per_sm=8, pipelines=3, max_wave_roots=20000))
    else:
        be = serve.PlainBackend(ctx, arena, pool_scene)
    out = serve.ServeLoop(reqs, be, budget).run()
    sums = dict(be.checksums)
    be.close()
    ctx.close()
    arena.close()
    torch.cuda.synchronize()
    return out, sums


def test_served_equals_plain():
    pool = _pool()
    reqs = serve.request_stream(pool, duration_s=3.0, rate=20.0, side_range=(128, 256), spps=(1, 4), recent=8,
                                rerender_spp=4)
    assert any(r.kind == "rerender" for r in reqs)
    budget = 3 * serve.scene_bytes_estimate(250000)   # evictions happen
    out_p, sums_p = _serve("plain", reqs, pool, budget)
    out_b, sums_b = _serve("batched", reqs, pool, budget)
    assert len(sums_b) == len(reqs) == len(sums_p)
    diff = [i for i in range(len(reqs)) if sums_b[i] != sums_p[i]]
    assert not diff, f"requests {diff[:10]} differ between the served mix and one render per launch"
    assert out_b["latency_p99_s"] >= out_b["latency_p50_s"] >= 0


def test_c_abi_server_equals_plain():
    """mrt_serve_* (the served form for a C/C++ host): requests submitted at their arrival times while
    others render, scenes admitted by footprint and evicted (their images kept for re-renders), every
    result equal to one mrt_render per request in arrival order."""
    import ctypes
    import time
    pool = _pool()
    reqs = serve.request_stream(pool, duration_s=2.0, rate=20.0, side_range=(128, 256), spps=(1, 4), recent=8,
                                rerender_spp=4)
    assert any(r.kind == "rerender" for r in reqs)
    hosts = {}

    def host(r):
        if r.geometry not in hosts:
            hosts[r.geometry] = pool[r.geometry].scene()
        return hosts[r.geometry]

    # one mrt_render per request, each scene's image kept between its requests
    ctx = m.Context(0)
    built, images, want = {}, {}, {}
    for r in reqs:
        if r.scene not in built:
            built[r.scene] = m.Scene(ctx, host(r)).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
        bm = images.setdefault(r.scene, np.zeros((r.side, r.side), np.uint32))
        built[r.scene].render(scenes.cli_camera(r.side, r.side), serve.request_opts(r), bitmap=bm)
        want[r.index] = bm.copy()
    for s in built.values():
        s.close()
    ctx.close()
    # the same stream through the C ABI
    lib = capi.load()
    o = capi.MrtServeOpts()
    o.budget_bytes = 3 * serve.scene_bytes_estimate(250000)    # evictions happen
    o.build_slack_bytes = 64 << 20
    o.batch.max_depth, o.batch.max_spl, o.batch.wave_roots, o.batch.max_wave_roots = 6, 1, 20000, 20000
    o.batch.block_threads, o.batch.blocks_per_sm, o.batch.pipelines = 128, 8, 3
    h = ctypes.c_void_p()
    assert lib.mrt_serve_create(0, ctypes.byref(o), ctypes.byref(h)) == capi.MRT_OK
    descs, sids = {}, {}
    accel = capi.MrtAccelOpts()
    accel.accelerator, accel.bvh_mode = capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST
    for r in reqs:
        if r.scene not in sids:
            descs[r.scene] = host(r).desc()
            sid = ctypes.c_uint64()
            assert lib.mrt_serve_add_scene(h, ctypes.byref(descs[r.scene]), ctypes.byref(accel), ctypes.byref(sid)) == 0
            sids[r.scene] = sid.value
    got = {r.index: np.zeros((r.side, r.side), np.uint32) for r in reqs}
    by_id = {}
    done = (ctypes.c_uint64 * 64)()
    n = ctypes.c_uint32()
    finished = set()
    t0 = time.perf_counter()
    k = 0
    while len(finished) < len(reqs):
        now = time.perf_counter() - t0
        while k < len(reqs) and reqs[k].arrival <= now:
            r = reqs[k]
            rid = ctypes.c_uint64()
            cam = scenes.cli_camera(r.side, r.side)
            opts = serve.request_opts(r)
            st = lib.mrt_serve_submit(h, sids[r.scene], ctypes.byref(cam), ctypes.byref(opts),
                                      got[r.index].ctypes.data_as(ctypes.c_void_p), ctypes.byref(rid))
            assert st == 0, lib.mrt_serve_error(h)
            by_id[rid.value] = r.index
            k += 1
        assert lib.mrt_serve_poll(h, done, 64, ctypes.byref(n)) == 0, lib.mrt_serve_error(h)
        finished.update(by_id[done[j]] for j in range(n.value))
        assert time.perf_counter() - t0 < 120
    st = capi.MrtServeStats()
    lib.mrt_serve_stats(h, ctypes.byref(st))
    lat = ctypes.c_double()
    assert lib.mrt_serve_request_latency(h, 1, ctypes.byref(lat)) == 0 and lat.value >= 0
    lib.mrt_serve_destroy(h)
    assert st.completed == len(reqs) and st.evictions > 0 and st.builds >= len(sids)
    diff = [i for i in range(len(reqs)) if not np.array_equal(got[i], want[i])]
    assert not diff, f"requests {diff[:10]} differ between the C-ABI server and one render per request"
