"""The batched renderer (mrt_batch_*) against the one-frame renderer and the oracle (GPU).

Every job of a batch must leave its bitmap and fp32 sums bit for bit as mrt_render with the same
arguments leaves them, whatever else shares its waves: mixed shaders, scenes with planes and
spheres, sample counts that do not divide the wave size (a pixel's samples then straddle two
waves), progressive continuation (spp_offset > 0 on a bitmap that already holds a running mean),
and waves cut from many jobs at once.
"""
import numpy as np
import pytest

import orc as O
from mobileraytracer_b200 import Batch, MrtError, Scene, capi, scenes

pytestmark = pytest.mark.gpu

NS, WH, PT = capi.MRT_SHADER_NOSHADOWS, capi.MRT_SHADER_WHITTED, capi.MRT_SHADER_PATHTRACER
H, S, R = capi.MRT_SAMPLER_HALTON, capi.MRT_SAMPLER_STRATIFIED, capi.MRT_SAMPLER_RANDOM


def _torch():
    import torch
    return torch


def job_list():
    """(host scene, camera, opts, initial-bitmap seed or None, with sums)."""
    cb = scenes.cornell_box()
    gr = scenes.glass_room()
    soup = scenes.triangle_soup(20000, 5, 160, 96)
    hf = scenes.heightfield(cells=48, seed=2)
    jobs = [
        (cb, cb.camera, capi.render_opts(shader=WH, width=64, height=64, spp=1, seed=1), None, True),
        (gr, gr.camera, capi.render_opts(shader=PT, width=96, height=64, spp=3, spl=2, seed=7), None, True),
        (soup, soup.camera, capi.render_opts(shader=NS, width=160, height=96, spp=2, seed=4), None, False),
        (hf, hf.camera, capi.render_opts(shader=PT, width=80, height=48, spp=5, pixel_sampler=H, light_sampler=H,
                                         rr_sampler=H, depth_min=3, depth_max=6, seed=11), None, True),
        (cb, cb.camera, capi.render_opts(shader=PT, width=48, height=48, spp=4, pixel_sampler=S, light_sampler=S,
                                         rr_sampler=R, depth_min=2, depth_max=5, seed=9, spp_offset=4), 3, True),
        (gr, gr.camera, capi.render_opts(shader=WH, width=64, height=48, spp=2, spl=3, seed=2), None, False),
        (soup, soup.camera, capi.render_opts(shader=PT, width=64, height=64, spp=1, seed=8), None, True),
        (gr, scenes.orthographic((0.3, 0.2, -3.4), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 2.6, 1.9),
         capi.render_opts(shader=capi.MRT_SHADER_DEPTHMAP, width=64, height=48, spp=2, seed=5,
                          depth_point=(1.5, 1.0, 2.0)), None, True),
        (cb, cb.camera, capi.render_opts(shader=capi.MRT_SHADER_DIFFUSE, width=48, height=32, spp=3, seed=6), None, True),
    ]
    return jobs


def initial_bitmap(opts, seed):
    if seed is None:
        return np.zeros((opts.height, opts.width), np.uint32)
    rng = np.random.default_rng(seed)
    return rng.integers(0, 2 ** 32, size=(opts.height, opts.width), dtype=np.uint64).astype(np.uint32)


def plain_and_batched(ctx, batch_kwargs, repeat_jobs=1):
    torch = _torch()
    built = {}
    plain, batched, ids = [], [], []
    b = Batch(ctx, **batch_kwargs)
    rays = [0, 0]
    for rep in range(repeat_jobs):
        for k, (sc, cam, opts, bseed, with_acc) in enumerate(job_list()):
            key = id(sc)
            if key not in built:
                built[key] = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST,
                                                  camera_position=list(cam.position))
            g = built[key]
            bm0 = initial_bitmap(opts, bseed)
            acc0 = np.zeros((opts.height, opts.width, 4), np.float32)
            bm_p = torch.from_numpy(bm0.view(np.int32).copy()).cuda()
            acc_p = torch.from_numpy(acc0.copy()).cuda() if with_acc else None
            _, _, st = g.render(cam, opts, bitmap=bm_p, accum=acc_p)
            rays[0] += st.rays_closest
            rays[1] += st.rays_shadow
            bm_b = torch.from_numpy(bm0.view(np.int32).copy()).cuda()
            acc_b = torch.from_numpy(acc0.copy()).cuda() if with_acc else None
            ids.append(b.submit(g, cam, opts, bm_b, acc_b))
            plain.append((bm_p, acc_p))
            batched.append((bm_b, acc_b))
    b.run()
    done = b.completed()
    stats = b.stats()
    b.close()
    return plain, batched, ids, done, stats, rays


@pytest.mark.parametrize("kw", [
    dict(wave_roots=3001, block_threads=128, blocks_per_sm=8, pipelines=2),  # pixels straddle waves
    dict(wave_roots=1024, block_threads=64, blocks_per_sm=16, graph=False, pipelines=3),  # plain launches
    dict(wave_roots=5000, policy=capi.MRT_BATCH_FIFO, pipelines=1),
    dict(wave_roots=7777, policy=capi.MRT_BATCH_EQUAL_SHARE, pipelines=3),  # every job in every wave
    dict(wave_roots=2000, pipelines=4, block_threads=256, blocks_per_sm=4),  # 4 waves in flight
    dict(max_wave_roots=1 << 16),                                            # autotuned
    dict(wave_roots=3001, kernel=capi.MRT_BATCH_KERNEL_PATHS, pipelines=2),   # whole paths per lane
    dict(wave_roots=50000, kernel=capi.MRT_BATCH_KERNEL_PATHS, pipelines=4,
         policy=capi.MRT_BATCH_EQUAL_SHARE),
])
def test_batch_equals_plain(ctx, kw):
    plain, batched, ids, done, stats, rays = plain_and_batched(ctx, kw)
    for k, ((bp, ap), (bb, ab)) in enumerate(zip(plain, batched)):
        nd = int((bp != bb).sum())
        assert nd == 0, f"job {k}: {nd} bitmap pixels differ"
        if ap is not None:
            assert bool((ap == ab).all()), f"job {k}: sums differ"
    assert sorted(done) == sorted(ids)
    assert stats.jobs_done == len(ids) and stats.jobs_submitted == len(ids)
    assert (stats.rays_closest, stats.rays_shadow) == tuple(rays)
    assert stats.paths == sum(o.width * o.height * o.spp for _, _, o, _, _ in job_list())
    if kw.get("wave_roots") == 3001:
        assert stats.waves >= stats.paths // 3001
        assert stats.wave_roots == 3001 and (stats.autotuned == 0 or "kernel" in kw)
    if "max_wave_roots" in kw:
        assert stats.autotuned > 1 and stats.block_threads in (64, 128, 256) and 1 <= stats.pipelines <= 4
    if "pipelines" in kw:
        assert stats.pipelines == kw["pipelines"]
    if "kernel" in kw:
        assert stats.kernel == kw["kernel"]


def test_batch_many_jobs_share_waves(ctx):
    """Three copies of the job list in one batch: waves are cut from up to 21 jobs at once."""
    plain, batched, ids, done, stats, rays = plain_and_batched(
        ctx, dict(wave_roots=40000, policy=capi.MRT_BATCH_EQUAL_SHARE), repeat_jobs=3)
    for k, ((bp, ap), (bb, ab)) in enumerate(zip(plain, batched)):
        assert int((bp != bb).sum()) == 0, f"job {k}"
        if ap is not None:
            assert bool((ap == ab).all()), f"job {k}: sums differ"
    assert sorted(done) == sorted(ids)


def test_batch_job_matches_oracle(ctx):
    """A batched PathTracer job against the oracle directly (glass room: planes, spheres, glass)."""
    torch = _torch()
    sc = scenes.glass_room()
    opts = capi.render_opts(shader=PT, width=64, height=48, spp=2, spl=2, seed=5)
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, camera_position=list(sc.camera.position))
    b = Batch(ctx, wave_roots=2048, block_threads=128, blocks_per_sm=8)
    bm = torch.zeros((48, 64), dtype=torch.int32, device="cuda")
    acc = torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda")
    b.submit(g, sc.camera, opts, bm, acc)
    b.run()
    b.close()
    bm_o, acc_o, _ = O.OrcScene(sc, 3, camera_position=list(sc.camera.position)).render(sc.camera, opts)
    assert np.array_equal(bm.cpu().numpy().view(np.uint32), bm_o)
    assert float(np.abs(acc.cpu().numpy()[..., :3] - acc_o[..., :3]).max()) <= 1e-3


def test_batch_rejects(ctx):
    torch = _torch()
    sc = scenes.cornell_box()
    ref = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_REFERENCE, camera_position=list(sc.camera.position))
    fast = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, camera_position=list(sc.camera.position))
    b = Batch(ctx, wave_roots=1024, block_threads=128, blocks_per_sm=4, max_jobs=2, max_depth=4)
    bm = torch.zeros((64, 64), dtype=torch.int32, device="cuda")
    with pytest.raises(MrtError) as e:
        b.submit(ref, sc.camera, capi.render_opts(shader=WH, width=64, height=64), bm)
    assert e.value.status == capi.MRT_ERR_ARG
    with pytest.raises(MrtError) as e:   # 40 is not a multiple of 16
        b.submit(fast, sc.camera, capi.render_opts(shader=WH, width=40, height=64), bm)
    assert e.value.status == capi.MRT_ERR_ARG
    with pytest.raises(MrtError) as e:   # depth above the batch's ray pool
        b.submit(fast, sc.camera, capi.render_opts(shader=PT, width=64, height=64, depth_max=8), bm)
    assert e.value.status == capi.MRT_ERR_ARG
    with pytest.raises(MrtError):        # host buffers
        b.submit(fast, sc.camera, capi.render_opts(shader=WH, width=64, height=64), np.zeros((64, 64), np.uint32))
    o = capi.render_opts(shader=WH, width=64, height=64, depth_max=4)
    bms = [torch.zeros((64, 64), dtype=torch.int32, device="cuda") for _ in range(3)]
    b.submit(fast, sc.camera, o, bms[0])
    b.submit(fast, sc.camera, o, bms[1])
    with pytest.raises(MrtError) as e:   # two slots, both outstanding
        b.submit(fast, sc.camera, o, bms[2])
    assert e.value.status == capi.MRT_ERR_LIMIT
    b.run()
    b.completed()
    b.submit(fast, sc.camera, o, bms[2])   # slots free again
    b.run()
    assert len(b.completed()) == 1
    assert bool((bms[0] == bms[2]).all()) and bool((bms[0] == bms[1]).all())
    b.close()
