"""mrt_render_noalloc: the render entry point for callers that cannot allocate device memory while
they render (processes whose device memory belongs to another allocator or a fixed budget,
latency-critical threads that must not meet cudaMalloc's implicit synchronisation).  It keeps its scratch in one static device
array instead of allocating, so it must produce exactly what mrt_render produces for the same device
buffers, call after call (the array keeps the previous call's contents), and refuse requests
beyond its fixed limits.  This file is collected last so a failure here comes after every other
test has run."""
import ctypes

import numpy as np
import pytest

from mobileraytracer_b200 import Scene, capi, scenes

pytestmark = pytest.mark.gpu


def _noalloc(scene, cam, opts, bitmap, accum):
    stats = capi.MrtRenderStats()
    st = scene.lib.mrt_render_noalloc(scene.h, ctypes.byref(cam), ctypes.byref(opts), ctypes.c_void_p(bitmap.data_ptr()),
                                      opts.width * 4, ctypes.c_void_p(accum.data_ptr()), ctypes.byref(stats))
    return st, stats


CASES = [
    ("glass_room", capi.MRT_SHADER_PATHTRACER, capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, 3, 2),
    ("glass_room", capi.MRT_SHADER_WHITTED, capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST, 2, 2),
    ("cornell_box", capi.MRT_SHADER_PATHTRACER, capi.MRT_ACCEL_BVH, capi.MRT_BVH_REFERENCE, 4, 1),
    ("soup", capi.MRT_SHADER_NOSHADOWS, capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, 2, 1),
    # the direct shaders on the accelerators without the persistent engine (one thread per pixel)
    ("soup", capi.MRT_SHADER_NOSHADOWS, capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST, 2, 1),
    ("glass_room", capi.MRT_SHADER_DEPTHMAP, capi.MRT_ACCEL_BVH, capi.MRT_BVH_REFERENCE, 1, 1),
    ("cornell_box", capi.MRT_SHADER_DIFFUSE, capi.MRT_ACCEL_NAIVE, capi.MRT_BVH_FAST, 1, 1),
]


@pytest.mark.parametrize("name,shader,accel,mode,spp,spl", CASES)
def test_noalloc_matches_mrt_render_twice(ctx, name, shader, accel, mode, spp, spl):
    import torch
    sc = {"glass_room": scenes.glass_room, "cornell_box": scenes.cornell_box,
          "soup": lambda: scenes.triangle_soup(20000, 5, 128, 96)}[name]()
    w, h = 128, 96   # 96 rows = 16 blocks of 6: the plain-rectangle schedule
    g = Scene(ctx, sc).build(accel, mode)
    for call, seed in enumerate((11, 11, 12)):   # two identical calls in a row, then another stream
        opts = capi.render_opts(shader=shader, width=w, height=h, spp=spp, spl=spl, seed=seed, depth_min=3, depth_max=6)
        want_bm = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        want_acc = torch.zeros(w * h * 4, dtype=torch.float32, device="cuda")
        g.render(sc.camera, opts, bitmap=want_bm, accum=want_acc)
        got_bm = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        got_acc = torch.zeros(w * h * 4, dtype=torch.float32, device="cuda")
        st, stats = _noalloc(g, sc.camera, opts, got_bm, got_acc)
        assert st == capi.MRT_OK, g.lib.mrt_context_error(ctx.h)
        torch.cuda.synchronize()
        tol = 1e-3 if shader == capi.MRT_SHADER_PATHTRACER else 1e-4
        assert float((got_acc - want_acc).abs().max()) <= tol, (name, call)
        assert torch.equal(got_bm, want_bm), (name, call)
        assert stats.paths == w * h * spp and stats.rays_closest >= w * h * spp


def test_noalloc_rejects_requests_beyond_its_limits(ctx):
    import torch
    sc = scenes.glass_room()
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH)
    bm = torch.zeros(128 * 96, dtype=torch.int32, device="cuda")
    acc = torch.zeros(128 * 96 * 4, dtype=torch.float32, device="cuda")
    too_many_light_samples = capi.render_opts(shader=capi.MRT_SHADER_WHITTED, width=128, height=96, spl=5)
    too_deep = capi.render_opts(shader=capi.MRT_SHADER_PATHTRACER, width=128, height=96, depth_max=11)
    odd_width = capi.render_opts(shader=capi.MRT_SHADER_WHITTED, width=100, height=96)
    for opts in (too_many_light_samples, too_deep):
        st, _ = _noalloc(g, sc.camera, opts, bm, acc)
        assert st == capi.MRT_ERR_ARG
    st = g.lib.mrt_render_noalloc(g.h, ctypes.byref(sc.camera), ctypes.byref(odd_width), ctypes.c_void_p(bm.data_ptr()),
                                  100 * 4, ctypes.c_void_p(acc.data_ptr()), None)
    assert st == capi.MRT_ERR_ARG
    # the context stays usable after the refusals
    ok, _ = _noalloc(g, sc.camera, capi.render_opts(shader=capi.MRT_SHADER_WHITTED, width=128, height=96), bm, acc)
    assert ok == capi.MRT_OK
