"""Whole-frame parity of mrt_render (Renderer::renderFrame on the device) against the oracle's
restatement of the renderer with the same keyed sample stream (GPU).

NoShadows, Whitted and PathTracer frames must equal the oracle bit for bit: the ARGB8888 bitmap
(incrementalAvg of every sample, Utils.cpp:48-70) and the fp32 per-pixel sums.  The tolerance the
specification allows (1e-4 for the deterministic shaders, 1e-3 for PathTracer radiance) is asserted
on the fp32 sums as the documented bound; the bitmaps are compared exactly.
"""
import os

import numpy as np
import pytest

import orc as O
from mobileraytracer_b200 import Scene, capi, scenes

pytestmark = pytest.mark.gpu

NS, WH, PT = capi.MRT_SHADER_NOSHADOWS, capi.MRT_SHADER_WHITTED, capi.MRT_SHADER_PATHTRACER
GPU_ACCELS = [  # (gpu accelerator, bvh mode, oracle accelerator with the same answers)
    (capi.MRT_ACCEL_NAIVE, capi.MRT_BVH_FAST, 0),
    (capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST, 1),
    (capi.MRT_ACCEL_BVH, capi.MRT_BVH_REFERENCE, 2),
    (capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, 3),
]


def render_both(ctx, sc, cam, opts, accel, mode, oacc):
    g = Scene(ctx, sc).build(accel, mode, camera_position=list(cam.position))
    bm_g, acc_g, stats = g.render(cam, opts, accum=np.zeros((opts.height, opts.width, 4), np.float32))
    o = O.OrcScene(sc, oacc, camera_position=list(cam.position))
    bm_o, acc_o, counts = o.render(cam, opts)
    return bm_g, acc_g, stats, bm_o, acc_o, counts


def assert_same(bm_g, acc_g, bm_o, acc_o, tol):
    diff = np.abs(acc_g[..., :3] - acc_o[..., :3])
    assert float(diff.max()) <= tol, f"max |radiance difference| {diff.max()}"
    nd = int(np.sum(bm_g != bm_o))
    assert nd == 0, f"{nd} bitmap pixels differ (max radiance diff {diff.max()})"


@pytest.mark.parametrize("accel,mode,oacc", GPU_ACCELS)
def test_noshadows_soup(ctx, accel, mode, oacc):
    sc = scenes.triangle_soup(30000, 2, 320, 240)
    opts = capi.render_opts(shader=NS, width=320, height=240, spp=1, spl=1)
    bm_g, acc_g, stats, bm_o, acc_o, counts = render_both(ctx, sc, sc.camera, opts, accel, mode, oacc)
    assert_same(bm_g, acc_g, bm_o, acc_o, 1e-4)
    assert stats.rays_closest == counts[0]


@pytest.mark.parametrize("shader", [NS, WH, PT])
@pytest.mark.parametrize("accel,mode,oacc", GPU_ACCELS)
def test_glass_room_all_shaders(ctx, shader, accel, mode, oacc):
    """planes + spheres (mirror, glass ior 1.9, diffuse+specular) + triangles + 2 area lights."""
    sc = scenes.glass_room()
    opts = capi.render_opts(shader=shader, width=96, height=64, spp=3, spl=2, seed=7)
    bm_g, acc_g, stats, bm_o, acc_o, counts = render_both(ctx, sc, sc.camera, opts, accel, mode, oacc)
    assert_same(bm_g, acc_g, bm_o, acc_o, 1e-3 if shader == PT else 1e-4)
    assert stats.rays_closest == counts[0] and stats.rays_shadow == counts[1]


def test_cornell_whitted_256(ctx):
    """Cornell box, Whitted, 256x256, 1 spp, Constant(0.5) camera sampler, BVH."""
    sc = scenes.cornell_box()
    opts = capi.render_opts(shader=WH, width=256, height=256, spp=1, spl=1, seed=1)
    for accel, mode, oacc in ((capi.MRT_ACCEL_BVH, capi.MRT_BVH_REFERENCE, 2), (capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, 3)):
        bm_g, acc_g, stats, bm_o, acc_o, counts = render_both(ctx, sc, sc.camera, opts, accel, mode, oacc)
        assert_same(bm_g, acc_g, bm_o, acc_o, 1e-4)
        assert np.count_nonzero(bm_g & 0xFFFFFF) > 256 * 256 // 2


@pytest.mark.parametrize("sampler", [capi.MRT_SAMPLER_STRATIFIED, capi.MRT_SAMPLER_HALTON, capi.MRT_SAMPLER_RANDOM])
def test_pathtracer_samplers_rr(ctx, sampler):
    """PathTracer with Russian roulette beyond depth 3, max depth 6 (the terrain frame's setting) and every
    sampler kind on the camera jitter, the light positions and the roulette."""
    sc = scenes.cornell_box()
    opts = capi.render_opts(shader=PT, width=64, height=64, spp=8, spl=1, pixel_sampler=sampler,
                            light_sampler=sampler, rr_sampler=sampler, depth_min=3, depth_max=6, seed=3)
    bm_g, acc_g, stats, bm_o, acc_o, counts = render_both(ctx, sc, sc.camera, opts, capi.MRT_ACCEL_BVH,
                                                          capi.MRT_BVH_FAST, 3)
    assert_same(bm_g, acc_g, bm_o, acc_o, 1e-3)


def test_terrain_pathtracer_crop(ctx):
    """The terrain scene (524,288-triangle fBm terrain, 4 area quads) at 64x64, 4 spp HaltonSeq,
    depth 6, RR after 3: per-pixel radiance within 1e-3 of the oracle (asserted: exact)."""
    sc = scenes.heightfield(512, 1, width=64, height=64)
    opts = capi.render_opts(shader=PT, width=64, height=64, spp=4, spl=1, pixel_sampler=capi.MRT_SAMPLER_HALTON,
                            light_sampler=capi.MRT_SAMPLER_HALTON, rr_sampler=capi.MRT_SAMPLER_HALTON,
                            depth_min=3, depth_max=6, seed=1)
    bm_g, acc_g, stats, bm_o, acc_o, counts = render_both(ctx, sc, sc.camera, opts, capi.MRT_ACCEL_BVH,
                                                          capi.MRT_BVH_FAST, 3)
    assert_same(bm_g, acc_g, bm_o, acc_o, 1e-3)


def test_progressive_continuation(ctx):
    """spp_offset continues the stream and the running mean: 2 + 2 samples == 4 samples."""
    sc = scenes.glass_room()
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH)
    o4 = capi.render_opts(shader=PT, width=48, height=48, spp=4, spl=1, seed=5)
    bm4, _, _ = g.render(sc.camera, o4)
    bm = np.zeros((48, 48), np.uint32)
    g.render(sc.camera, capi.render_opts(shader=PT, width=48, height=48, spp=2, spl=1, seed=5), bitmap=bm)
    o2b = capi.render_opts(shader=PT, width=48, height=48, spp=2, spl=1, seed=5, spp_offset=2)
    o2b.spp = 2
    # the stratified count must be the full render's for Stratified; Random/Constant do not use it
    g.render(sc.camera, o2b, bitmap=bm)
    assert (bm == bm4).all()


def test_odd_sizes_and_stride(ctx):
    """Width not a multiple of 16 (blocks overlap / leave gaps exactly as the reference's block
    arithmetic does) and a padded row pitch."""
    sc = scenes.glass_room()
    for w, h in ((100, 50), (37, 29)):
        for shader in (NS, WH):
            opts = capi.render_opts(shader=shader, width=w, height=h, spp=2, spl=1, seed=2)
            bm_g, acc_g, _, bm_o, acc_o, _ = render_both(ctx, sc, sc.camera, opts, capi.MRT_ACCEL_BVH,
                                                         capi.MRT_BVH_REFERENCE, 2)
            assert (bm_g == bm_o).all(), (w, h, shader)
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH)
    opts = capi.render_opts(shader=NS, width=64, height=32, spp=1)
    padded = np.full((32, 80), 0xDEADBEEF, np.uint32)
    g.render(sc.camera, opts, bitmap=padded, stride_bytes=80 * 4)
    plain, _, _ = g.render(sc.camera, opts)
    assert (padded[:, :64] == plain).all() and (padded[:, 64:] == 0xDEADBEEF).all()


def test_host_path_keeps_unrendered_rows(ctx):
    """Host buffers: a first pass (spp_offset 0) copies in only the rows below the block schedule,
    since it overwrites the rest without reading it; a continuation (spp_offset > 0) reads them all.
    Either way the host result equals the device path started from the same bitmap."""
    torch = pytest.importorskip("torch")
    sc = scenes.glass_room()
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH)
    # 152 = 16 * 9 + 8 with 152 / 9 = 16 blocks down: the plain rectangle of rows 0..143; rows
    # 144..151 are not rendered (as rows 1072..1079 of a 1080-row frame)
    w, h = 96, 152
    rng = np.random.default_rng(3)
    start = rng.integers(0, 2**32, size=(h, w), dtype=np.uint32)
    for shader, spp_offset in ((NS, 0), (PT, 0), (NS, 1), (PT, 2)):
        opts = capi.render_opts(shader=shader, width=w, height=h, spp=2, spl=1, seed=7, spp_offset=spp_offset)
        host = start.copy()
        g.render(sc.camera, opts, bitmap=host)
        dev = torch.from_numpy(start.view(np.int32).copy()).cuda()
        g.render(sc.camera, opts, bitmap=dev)
        torch.cuda.synchronize()
        assert (host == dev.cpu().numpy().view(np.uint32)).all(), (shader, spp_offset)
        assert (host[144:] == start[144:]).all()
        assert (host[:144] != start[:144]).any()
    g.close()


def test_host_path_trace_and_shade_equal_the_device_path(ctx):
    """Host buffers on the NoShadows trace + shade path: bitmap and sums equal the device path on the
    FAST BVH and the RegularGrid, for an odd width (row-major tasks), several samples per pixel, and with
    a padded row pitch."""
    torch = pytest.importorskip("torch")
    soup = scenes.triangle_soup(20_000, 5, 320, 240)
    for accel, w, h, spp in ((capi.MRT_ACCEL_BVH, 320, 240, 1), (capi.MRT_ACCEL_BVH, 97, 200, 3),
                             (capi.MRT_ACCEL_REGULAR_GRID, 320, 240, 2)):
        g = Scene(ctx, soup).build(accel)
        opts = capi.render_opts(shader=NS, width=w, height=h, spp=spp, spl=1, seed=9)
        host_bm = np.full((h, w), 0x12345678, np.uint32)
        host_acc = np.zeros((h, w, 4), np.float32)
        _, _, st = g.render(soup.camera, opts, bitmap=host_bm, accum=host_acc)
        assert st.kernel_launches >= 2 and st.kernel_launches % 2 == 0   # trace and shade passes
        dev_bm = torch.full((h * w,), 0x12345678, dtype=torch.int32, device="cuda")
        dev_acc = torch.zeros(h * w * 4, dtype=torch.float32, device="cuda")
        g.render(soup.camera, opts, bitmap=dev_bm, accum=dev_acc)
        torch.cuda.synchronize()
        assert np.array_equal(host_bm, dev_bm.cpu().numpy().view(np.uint32).reshape(h, w)), (accel, w, h)
        assert np.array_equal(host_acc.view(np.uint32), dev_acc.cpu().numpy().view(np.uint32).reshape(h, w, 4))
        # a padded row pitch (the block schedule then depends on the pitch, Renderer.cpp:82-93): one copy
        # at the end, the same bitmap as the device path with that pitch
        pitch = w + 3
        padded = np.full((h, pitch), 0x12345678, np.uint32)
        g.render(soup.camera, opts, bitmap=padded, stride_bytes=4 * pitch)
        dev_pad = torch.full((h * pitch,), 0x12345678, dtype=torch.int32, device="cuda")
        g.render(soup.camera, opts, bitmap=dev_pad, stride_bytes=4 * pitch)
        torch.cuda.synchronize()
        assert np.array_equal(padded, dev_pad.cpu().numpy().view(np.uint32).reshape(h, pitch))
        g.close()


def test_page_locked_host_frames_shade_in_bands(ctx):
    """Page-locked host buffers on the plain rectangle: the trace + shade path shades the last samples
    in bands of whole 16-row stripes and copies each out while the next is shaded.  Bitmap and sums
    equal the device path started from the same bytes (first passes and continuations, one and several
    samples, FAST BVH and RegularGrid), the rows below the block schedule keep the caller's bytes, and
    pageable buffers of the same frame give the same result in one shading launch per pass."""
    torch = pytest.importorskip("torch")
    soup = scenes.triangle_soup(20_000, 5, 320, 240)
    rng = np.random.default_rng(11)
    for accel, w, h, spp, spp_offset in ((capi.MRT_ACCEL_BVH, 320, 200, 1, 0), (capi.MRT_ACCEL_BVH, 320, 240, 3, 0),
                                         (capi.MRT_ACCEL_REGULAR_GRID, 320, 200, 2, 1),
                                         (capi.MRT_ACCEL_BVH, 96, 152, 2, 2)):
        g = Scene(ctx, soup).build(accel)
        opts = capi.render_opts(shader=NS, width=w, height=h, spp=spp, spl=1, seed=4, spp_offset=spp_offset)
        start = rng.integers(0, 2**32, size=(h, w), dtype=np.uint32)
        start_acc = rng.random((h, w, 4), dtype=np.float32)
        host_bm = torch.from_numpy(start.view(np.int32).copy()).pin_memory().numpy().view(np.uint32)
        host_acc = torch.from_numpy(start_acc.copy()).pin_memory().numpy()
        _, _, st = g.render(soup.camera, opts, bitmap=host_bm, accum=host_acc)
        rows = 16 * (h // 16)
        assert st.kernel_launches > 2, (accel, w, h)   # one trace launch, several shading bands
        dev_bm = torch.from_numpy(start.view(np.int32).copy()).cuda()
        dev_acc = torch.from_numpy(start_acc.copy()).cuda()
        g.render(soup.camera, opts, bitmap=dev_bm, accum=dev_acc)
        torch.cuda.synchronize()
        assert np.array_equal(host_bm, dev_bm.cpu().numpy().view(np.uint32)), (accel, w, h, spp)
        assert np.array_equal(host_acc.view(np.uint32), dev_acc.cpu().numpy().view(np.uint32))
        assert (host_bm[rows:] == start[rows:]).all() and (host_acc[rows:] == start_acc[rows:]).all()
        pageable = start.copy()
        pageable_acc = start_acc.copy()
        _, _, st2 = g.render(soup.camera, opts, bitmap=pageable, accum=pageable_acc)
        assert np.array_equal(pageable, host_bm) and np.array_equal(pageable_acc.view(np.uint32), host_acc.view(np.uint32))
        assert st2.kernel_launches < st.kernel_launches
        g.close()


def test_errors_are_reported(ctx):
    import mobileraytracer_b200 as m
    sc = scenes.glass_room()
    g = Scene(ctx, sc)
    with pytest.raises(m.MrtError) as e:
        g.render(sc.camera, capi.render_opts(width=32, height=32))
    assert e.value.status == capi.MRT_ERR_STATE
    g.build(capi.MRT_ACCEL_BVH)
    with pytest.raises(m.MrtError) as e:
        g.render(sc.camera, capi.render_opts(width=8, height=8))
    assert e.value.status == capi.MRT_ERR_ARG
    bad = capi.render_opts(width=32, height=32)
    bad.shader = 9
    with pytest.raises(m.MrtError):
        g.render(sc.camera, bad)
    ok, _, _ = g.render(sc.camera, capi.render_opts(width=32, height=32))   # context still usable
    assert ok.any()


@pytest.mark.parametrize("shader", [capi.MRT_SHADER_DEPTHMAP, capi.MRT_SHADER_DIFFUSE, NS])
@pytest.mark.parametrize("ortho", [False, True])
@pytest.mark.parametrize("accel,mode,oacc", GPU_ACCELS)
def test_depthmap_diffuse_orthographic(ctx, shader, ortho, accel, mode, oacc):
    """DepthMap (DepthMap.cpp:19-26) and DiffuseMaterial (DiffuseMaterial.cpp:16-38) frames, and the
    Orthographic camera (Orthographic.cpp:23-46, including its film rectangle in the grid bounds)."""
    sc = scenes.glass_room()
    cam = scenes.orthographic((0.3, 0.2, -3.4), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 2.6, 1.9) if ortho else sc.camera
    sc.camera = cam
    opts = capi.render_opts(shader=shader, width=96, height=64, spp=2, spl=1, seed=3, depth_point=(1.5, 1.0, 2.0),
                            pixel_sampler=capi.MRT_SAMPLER_STRATIFIED)
    g = Scene(ctx, sc).build(accel, mode, camera=cam)
    bm_g, acc_g, stats = g.render(cam, opts, accum=np.zeros((opts.height, opts.width, 4), np.float32))
    bm_o, acc_o, counts = O.OrcScene(sc, oacc, camera=cam).render(cam, opts)
    assert_same(bm_g, acc_g, bm_o, acc_o, 1e-4)
    assert stats.rays_closest == counts[0]
    assert np.count_nonzero(bm_g & 0xFFFFFF) > 1000


def test_stop_and_progress(ctx):
    """Renderer::stopRender from another thread while renderFrame runs (Renderer.cpp:61-65) and
    getSample as progress (Renderer.cpp:118-120): the render returns MRT_ERR_CANCELLED after the
    waves already queued, having reported progress, and the scene renders normally afterwards."""
    import threading
    import time
    import torch
    from mobileraytracer_b200 import MrtError
    sc = scenes.cornell_box()
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    opts = capi.render_opts(shader=PT, width=512, height=512, spp=512, spl=1, depth_min=3, depth_max=6)
    bm = torch.zeros(512 * 512, dtype=torch.int32, device="cuda")
    box = {}

    def run():
        try:
            g.render(sc.camera, opts, bitmap=bm)
            box["status"] = capi.MRT_OK
        except MrtError as e:
            box["status"] = e.status

    t = threading.Thread(target=run)
    t.start()
    seen = 0
    t0 = time.time()
    while t.is_alive() and time.time() - t0 < 60:
        seen = max(seen, g.progress())
        if seen > 0:
            g.stop()
            break
        time.sleep(0.001)
    t.join(120)
    assert not t.is_alive()
    assert box["status"] == capi.MRT_ERR_CANCELLED, box
    assert 0 < seen < 512
    small = capi.render_opts(shader=PT, width=64, height=64, spp=2, spl=1)
    g.render(sc.camera, small)   # no error: the stop request was consumed


def test_whole_paths_equal_wavefront(ctx, tmp_path):
    """The same PathTracer and Whitted frames from whole-path launches (small frames, this process)
    and from the level-by-level wavefront (a process with MRT_PATHS_MAX=0)."""
    import subprocess
    import sys
    code = (
        "import sys, numpy as np\n"
        "sys.path.insert(0, %r)\n"
        "import mobileraytracer_b200 as m\n"
        "from mobileraytracer_b200 import capi, scenes\n"
        "ctx = m.Context(0)\n"
        "out = []\n"
        "for sh in (1, 2):\n"
        "    sc = scenes.glass_room()\n"
        "    o = capi.render_opts(shader=sh, width=96, height=64, spp=3, spl=2, seed=7)\n"
        "    g = m.Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)\n"
        "    bm, acc, st = g.render(sc.camera, o, accum=np.zeros((64, 96, 4), np.float32))\n"
        "    out += [bm, acc, np.array([st.rays_closest, st.rays_shadow], np.uint64)]\n"
        "np.savez(sys.argv[1], *out)\n" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),))
    path = str(tmp_path / "wf.npz")
    env = dict(os.environ, MRT_PATHS_MAX="0")
    r = subprocess.run([sys.executable, "-c", code, path], env=env, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    wf = np.load(path)
    for k, sh in enumerate((WH, PT)):
        sc = scenes.glass_room()
        o = capi.render_opts(shader=sh, width=96, height=64, spp=3, spl=2, seed=7)
        g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
        bm, acc, st = g.render(sc.camera, o, accum=np.zeros((64, 96, 4), np.float32))
        assert np.array_equal(bm, wf[f"arr_{3 * k}"])
        assert np.array_equal(acc.view(np.uint32), wf[f"arr_{3 * k + 1}"].view(np.uint32))
        assert [st.rays_closest, st.rays_shadow] == list(wf[f"arr_{3 * k + 2}"])


@pytest.mark.parametrize("shader", [WH, PT])
def test_glass_room_wavefront_with_material_queues(ctx, shader):
    """A frame above the whole-path limit (768x768 = 589,824 camera paths) of a scene that mixes
    diffuse walls with mirror and glass spheres, rendered with MRT_RENDER_SHADE_QUEUES: the FAST-BVH
    wavefront sorts every window of a level's rays by material class before shading.  The result
    equals the oracle bit for bit."""
    sc = scenes.glass_room()
    opts = capi.render_opts(shader=shader, width=768, height=768, spp=1, spl=1, seed=4,
                            flags=capi.MRT_RENDER_SHADE_QUEUES)
    bm_g, acc_g, stats, bm_o, acc_o, counts = render_both(ctx, sc, sc.camera, opts, capi.MRT_ACCEL_BVH,
                                                          capi.MRT_BVH_FAST, 3)
    assert_same(bm_g, acc_g, bm_o, acc_o, 1e-3 if shader == PT else 1e-4)
    assert stats.rays_closest == counts[0] and stats.rays_shadow == counts[1]
