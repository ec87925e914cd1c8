"""Parity at the sizes the benchmarks time (GPU).

* The 1920x1080 NoShadows frame of the 1,000,000-triangle soup through mrt_render on the FAST BVH
  (the trace and shade kernels the benchmark times) against the oracle's exact closest hit, on every
  97th pixel of the rows the block schedule renders (0..1071), plus the untouched rows 1072..1079
  (Renderer.cpp:20-21).
* The same frame on the RegularGrid (G = 128) against the oracle's reference walk.
* The reference BVH (BVH<Triangle>::trace, BVH.hpp:158-213, compiled from the reference sources) on
  the same camera rays: every ray where its closest hit differs from the exact one is classified
  (a box its slab test rejects although a closer triangle inside passes the reference's own
  triangle test, AABB.cpp:15-35; a near-tie within 1e-6 relative; other).  Only the first two kinds
  may occur.
* The 1024x1024 terrain PathTracer frame at its 64 spp HaltonSeq, depth 6, roulette beyond 3: a
  128x128 crop of the full frame against the oracle's restatement, per sample.
* Image RMSE against a 4096-spp render: the device's 64-spp image and the reference renderer's own
  64-spp image (compiled reference, its urandom-seeded MersenneTwister samplers, as the CLI wires
  them, c_wrapper.cpp:436-455) have the same RMSE within a statistical bound.
"""
import ctypes
import os

import numpy as np
import pytest

import orc as O
from mobileraytracer_b200 import Scene, capi, scenes

from helpers import near_tie_mask

pytestmark = pytest.mark.gpu

W, H = 1920, 1080


@pytest.fixture(scope="module")
def soup():
    return scenes.triangle_soup(1_000_000, 0, W, H)


@pytest.fixture(scope="module")
def soup_subset():
    """every 97th pixel of rows 0..1071 (the rows the 16-row block schedule renders)"""
    return np.arange(0, W * 16 * (H // 16), 97, dtype=np.int64)


def _expected_bitmap(values, old):
    lib = O.orc()
    out = np.empty(len(values), np.uint32)
    v = np.ascontiguousarray(values, np.float32)
    for k in range(len(values)):
        out[k] = lib.orc_incremental_avg(O.fptr(v[k]), int(old[k]), 1)
    return out


def test_soup_1080p_frame_through_the_timed_kernel(ctx, soup, soup_subset):
    import torch
    opts = capi.render_opts(shader=capi.MRT_SHADER_NOSHADOWS, width=W, height=H, spp=1, spl=1)
    g = Scene(ctx, soup).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    bm = torch.full((H * W,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
    acc = torch.zeros(H * W * 4, dtype=torch.float32, device="cuda")
    _, _, st = g.render(soup.camera, opts, bitmap=bm, accum=acc)
    bm = bm.cpu().numpy().view(np.uint32).reshape(H, W)
    acc = acc.cpu().numpy().reshape(H, W, 4)
    assert st.rays_closest == W * 16 * (H // 16)
    # the rows below the block schedule keep the caller's bytes
    assert (bm[16 * (H // 16):] == 0x5A5A5A5A).all()
    o = O.OrcScene(soup, 3)
    xy = np.stack([soup_subset % W, soup_subset // W], 1).astype(np.uint32)
    vals = o.render_pixels(soup.camera, opts, xy, threads=os.cpu_count() or 8)[:, 0, :]
    ys, xs = soup_subset // W, soup_subset % W
    assert np.array_equal(acc[ys, xs, :3].view(np.uint32), vals.view(np.uint32))
    assert float(np.abs(acc[ys, xs, :3] - vals).max()) <= 1e-4   # the specification's bound, met exactly
    want = _expected_bitmap(vals, np.full(len(vals), 0x5A5A5A5A, np.uint32))
    nd = int(np.sum(bm[ys, xs] != want))
    assert nd == 0, f"{nd} of {len(want)} pixels differ"
    assert np.count_nonzero(bm[ys, xs] & 0xFFFFFF) > len(want) // 4   # the soup covers the frame's middle


def test_soup_1080p_frame_on_the_grid(ctx, soup, soup_subset):
    """The same frame on the RegularGrid at the reference's G = 128 (the grid trace and shade kernels the
    benchmark times): every 97th pixel equals the oracle's reference walk bit for bit."""
    import torch
    opts = capi.render_opts(shader=capi.MRT_SHADER_NOSHADOWS, width=W, height=H, spp=1, spl=1)
    g = Scene(ctx, soup).build(capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST)
    assert g.accel_info()["grid_size"] == 128
    bm = torch.zeros(H * W, dtype=torch.int32, device="cuda")
    acc = torch.zeros(H * W * 4, dtype=torch.float32, device="cuda")
    _, _, st = g.render(soup.camera, opts, bitmap=bm, accum=acc)
    assert st.kernel_launches == 2 and 0.0 < st.trace_ms <= st.device_ms
    bm = bm.cpu().numpy().view(np.uint32).reshape(H, W)
    acc = acc.cpu().numpy().reshape(H, W, 4)
    o = O.OrcScene(soup, capi.MRT_ACCEL_REGULAR_GRID, camera_position=list(soup.camera.position))
    xy = np.stack([soup_subset % W, soup_subset // W], 1).astype(np.uint32)
    vals = o.render_pixels(soup.camera, opts, xy, threads=os.cpu_count() or 8)[:, 0, :]
    ys, xs = soup_subset // W, soup_subset % W
    assert np.array_equal(acc[ys, xs, :3].view(np.uint32), vals.view(np.uint32))
    want = _expected_bitmap(vals, np.zeros(len(vals), np.uint32))
    assert int(np.sum(bm[ys, xs] != want)) == 0


def test_reference_bvh_disagreements_on_the_1080p_rays(ctx, soup, soup_subset):
    from mobileraytracer_b200 import camera as mcam
    rays = mcam.primary_rays(soup.camera, W, H, pixels=soup_subset[::2])
    g = Scene(ctx, soup).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    fast = g.trace_closest(rays)
    exact = O.OrcScene(soup, 3).trace_closest(rays, threads=os.cpu_count() or 8)
    ref = O.RefScene(soup, capi.MRT_ACCEL_BVH).trace_closest(rays, threads=os.cpu_count() or 8)
    # the product: exact closest hit, near-ties counted apart
    fast_diff = (fast["id"] != exact["id"]) | (fast["t"].view(np.uint32) != exact["t"].view(np.uint32))
    fast_ties = fast_diff & near_tie_mask(rays, fast, exact)
    assert int(np.sum(fast_diff & ~fast_ties)) == 0
    # the reference tree
    diff = (ref["id"] != exact["id"]) | (ref["t"].view(np.uint32) != exact["t"].view(np.uint32))
    ties = diff & near_tie_mask(rays, ref, exact)
    farther = diff & ~ties & (exact["id"] != capi.MRT_HIT_NONE) & (
        (ref["id"] == capi.MRT_HIT_NONE) | (ref["t"] > exact["t"]))
    # a farther (or missing) answer is a slab-test rejection only if the closer triangle passes the
    # reference's own triangle test at that distance
    lib = O.ref()
    confirmed = np.zeros(len(rays), bool)
    for k in np.nonzero(farther)[0]:
        idx = int(exact["id"][k]) & 0x3FFFFFFF
        abc = np.ascontiguousarray(soup.tri_abc[idx], np.float32)
        t = np.zeros(1, np.float32)
        hit = lib.ref_triangle_intersect(O.fptr(abc), None, None, O.fptr(rays["origin"][k].copy()),
                                         O.fptr(rays["direction"][k].copy()), ctypes.c_float(3.0e38), O.fptr(t),
                                         None, None)
        confirmed[k] = bool(hit) and t[0] == exact["t"][k]
    other = diff & ~ties & ~confirmed
    n = len(rays)
    print(f"\nreference BVH vs exact on {n} camera rays of the 1080p soup frame: {int(diff.sum())} differ = "
          f"{int(confirmed.sum())} slab-test rejections + {int(ties.sum())} near-ties + {int(other.sum())} other; "
          f"FAST: {int(fast_ties.sum())} near-ties, 0 other")
    assert int(other.sum()) == 0


def _terrain_opts(spp, sampler, depth_min=3, depth_max=6, seed=1, w=1024, h=1024):
    return capi.render_opts(shader=capi.MRT_SHADER_PATHTRACER, width=w, height=h, spp=spp, spl=1,
                            pixel_sampler=sampler, light_sampler=sampler, rr_sampler=sampler,
                            depth_min=depth_min, depth_max=depth_max, seed=seed)


def test_terrain_pathtracer_128_crop_at_64spp(ctx):
    import torch
    sc = scenes.heightfield(512, 1, width=1024, height=1024)
    opts = _terrain_opts(64, capi.MRT_SAMPLER_HALTON)
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    bm = torch.zeros(1024 * 1024, dtype=torch.int32, device="cuda")
    acc = torch.zeros(1024 * 1024 * 4, dtype=torch.float32, device="cuda")
    g.render(sc.camera, opts, bitmap=bm, accum=acc)
    bm = bm.cpu().numpy().view(np.uint32).reshape(1024, 1024)
    acc = acc.cpu().numpy().reshape(1024, 1024, 4)
    y0, x0 = 448, 448   # a 128x128 crop in the middle of the frame
    ys, xs = np.meshgrid(np.arange(y0, y0 + 128), np.arange(x0, x0 + 128), indexing="ij")
    xy = np.stack([xs.ravel(), ys.ravel()], 1).astype(np.uint32)
    vals = O.OrcScene(sc, 3).render_pixels(sc.camera, opts, xy, threads=os.cpu_count() or 8)   # (n, 64, 3)
    want_acc = np.zeros((len(xy), 3), np.float32)
    want_bm = np.zeros(len(xy), np.uint32)
    lib = O.orc()
    for s in range(opts.spp):   # the per-pixel sums and running mean in sample order
        want_acc += vals[:, s, :]
        v = np.ascontiguousarray(vals[:, s, :])
        for k in range(len(xy)):
            want_bm[k] = lib.orc_incremental_avg(O.fptr(v[k]), int(want_bm[k]), s + 1)
    got_acc = acc[ys.ravel(), xs.ravel(), :3]
    assert float(np.abs(got_acc - want_acc).max()) <= 1e-3 * opts.spp   # 1e-3 per sample (asserted: exact)
    assert np.array_equal(got_acc.view(np.uint32), want_acc.view(np.uint32))
    assert np.array_equal(bm[ys.ravel(), xs.ravel()], want_bm)
    assert (acc[ys.ravel(), xs.ravel(), 3] == opts.spp).all()


def _to_rgb(bitmap):
    b = bitmap.astype(np.uint32)
    return np.stack([b & 0xFF, (b >> 8) & 0xFF, (b >> 16) & 0xFF], -1).astype(np.float64) / 255.0


def test_terrain_rmse_against_4096spp_equals_the_reference_renderers(ctx):
    """128x128 terrain frames (the config's scene and camera) with the reference's compiled depth
    rule (RayDepthMin 4, RayDepthMax 8, Utils.hpp:34-35) so that the reference renderer as shipped
    computes the same estimator.  The 4096-spp image is the device path's fp32 mean (the
    parity-verified path); the 64-spp images are ARGB bitmaps (incrementalAvg), on both sides."""
    import torch
    w = h = 128
    sc = scenes.heightfield(512, 1, width=w, height=h)
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    ref_opts = _terrain_opts(4096, capi.MRT_SAMPLER_HALTON, 4, 8, seed=99, w=w, h=h)
    acc = torch.zeros(w * h * 4, dtype=torch.float32, device="cuda")
    g.render(sc.camera, ref_opts, bitmap=torch.zeros(w * h, dtype=torch.int32, device="cuda"), accum=acc)
    acc = acc.cpu().numpy().reshape(h, w, 4)
    truth = np.clip(acc[..., :3] / acc[..., 3:4], 0.0, 1.0)

    def rmse(bm):
        return float(np.sqrt(np.mean((_to_rgb(bm) - truth) ** 2)))

    gpu = {}
    for name, sampler in (("random", capi.MRT_SAMPLER_RANDOM), ("halton", capi.MRT_SAMPLER_HALTON)):
        vals = []
        for seed in (1, 2):
            bm, _, _ = g.render(sc.camera, _terrain_opts(64, sampler, 4, 8, seed=seed, w=w, h=h))
            vals.append(rmse(bm))
        gpu[name] = float(np.mean(vals))
    # the reference renderer as shipped: MersenneTwister samplers seeded from /dev/urandom, two runs
    cpu = []
    for _ in range(2):
        bm, _, _ = O.ref_render(sc, sc.camera, _terrain_opts(64, capi.MRT_SAMPLER_RANDOM, 4, 8, w=w, h=h),
                                capi.MRT_ACCEL_BVH, threads=os.cpu_count() or 8, fast=True)
        cpu.append(rmse(bm))
    cpu_rmse = float(np.mean(cpu))
    print(f"\nterrain 128x128, RMSE vs 4096 spp at 64 spp: device Random {gpu['random']:.5f}, device HaltonSeq "
          f"{gpu['halton']:.5f}, reference renderer (MersenneTwister, urandom) {cpu_rmse:.5f} "
          f"(runs {cpu[0]:.5f}, {cpu[1]:.5f})")
    # the same estimator with the same kind of sampler: equal RMSE up to sampling noise
    assert abs(gpu["random"] - cpu_rmse) <= 0.1 * cpu_rmse
    # the low-discrepancy sampler is no worse
    assert gpu["halton"] <= gpu["random"] * 1.05
