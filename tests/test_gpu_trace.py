"""Closest-hit / any-hit parity of the CUDA accelerators against the oracle (GPU).

NAIVE, REGULAR_GRID and BVH/REFERENCE walk the reference structures in the reference order, so the
hit id and the distance bits must equal the oracle's restatement of the same accelerator (itself
pinned to the reference's compiled code by test_oracle_vs_reference.py).  BVH/FAST must return the
Naive closest hit: same id and distance, near-ties (|dt| <= 1e-6 t) counted separately.
"""
import numpy as np
import pytest

import orc as O
from helpers import camera_rays, hits_equal, near_tie_mask, random_rays
from mobileraytracer_b200 import Scene, capi, scenes

pytestmark = pytest.mark.gpu

ACCELS = [
    ("naive", capi.MRT_ACCEL_NAIVE, capi.MRT_BVH_FAST, 0),
    ("grid", capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST, 1),
    ("bvh-reference", capi.MRT_ACCEL_BVH, capi.MRT_BVH_REFERENCE, 2),
]

SMALL_SCENES = {
    "glass_room": scenes.glass_room,
    "cornell_box": scenes.cornell_box,
    "soup20k": lambda: scenes.triangle_soup(20000, 3, 320, 240),
}


@pytest.mark.parametrize("scene_name", list(SMALL_SCENES))
@pytest.mark.parametrize("name,accel,mode,oacc", ACCELS)
def test_reference_accelerators_bit_exact(ctx, scene_name, name, accel, mode, oacc):
    sc = SMALL_SCENES[scene_name]()
    rays = random_rays(20000, seed=11)
    g = Scene(ctx, sc).build(accel, mode)
    o = O.OrcScene(sc, oacc)
    gh = g.trace_closest(rays)
    oh = o.trace_closest(rays)
    assert hits_equal(gh, oh).all(), f"{np.sum(~hits_equal(gh, oh))} of {len(rays)} rays differ"
    dist = np.full(len(rays), 0.6, np.float32)
    assert (g.trace_any(rays, dist) == o.trace_any(rays, dist)).all()


@pytest.mark.parametrize("scene_name", list(SMALL_SCENES))
def test_fast_bvh_equals_naive(ctx, scene_name):
    sc = SMALL_SCENES[scene_name]()
    rays = random_rays(20000, seed=12)
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    naive = O.OrcScene(sc, 0).trace_closest(rays)
    gh = g.trace_closest(rays)
    bad = ~hits_equal(gh, naive) & ~near_tie_mask(rays, gh, naive)
    assert not bad.any(), f"{bad.sum()} rays differ from the Naive closest hit"
    for d in (0.05, 0.6, 5.0):
        dist = np.full(len(rays), d, np.float32)
        assert (g.trace_any(rays, dist) == O.OrcScene(sc, 0).trace_any(rays, dist)).all()


def test_exclusion_and_secondary_rays(ctx):
    """Rays leaving a primitive must not hit it again (Ray::primitive_, Triangle.cpp:58)."""
    sc = scenes.glass_room()
    rays = random_rays(4000, seed=3)
    o = O.OrcScene(sc, 0)
    first = o.trace_closest(rays)
    hit = first["id"] != capi.MRT_HIT_NONE
    sec = rays[hit].copy()
    t = first["t"][hit].astype(np.float32)
    sec["origin"] = (sec["origin"] + sec["direction"] * t[:, None]).astype(np.float32)
    sec["exclude"] = first["id"][hit]
    sec["depth"] = 2
    for name, accel, mode, oacc in ACCELS:
        g = Scene(ctx, sc).build(accel, mode)
        assert hits_equal(g.trace_closest(sec), O.OrcScene(sc, oacc).trace_closest(sec)).all(), name
    gf = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST).trace_closest(sec)
    assert hits_equal(gf, o.trace_closest(sec)).all()


def test_degenerate_inputs(ctx):
    """Empty scene, zero-area triangles, axis-parallel and zero-component directions."""
    empty = scenes.Scene()
    empty.camera = scenes.camera((0, 0, -1), (0, 0, 1))
    rays = random_rays(256, seed=2)
    for accel, mode in ((0, 0), (1, 0), (2, 0), (2, 1)):
        h = Scene(ctx, empty).build(accel, mode).trace_closest(rays)
        assert (h["id"] == capi.MRT_HIT_NONE).all()
    sc = scenes.triangle_soup(3000, 9, 64, 64)
    sc.tri_abc[::7, 3:6] = sc.tri_abc[::7, 0:3]          # collapsed edge
    sc.tri_abc[::11, 6:9] = sc.tri_abc[::11, 3:6]
    axis = random_rays(3000, seed=4)
    axis["direction"][::3, 0] = 0.0
    axis["direction"][1::3, 1] = 0.0
    axis["direction"][2::3, 0:2] = 0.0
    axis["direction"][2::3, 2] = 1.0
    naive = O.OrcScene(sc, 0).trace_closest(axis)
    for accel, mode, oacc in ((0, 0, 0), (1, 0, 1), (2, 1, 2)):
        g = Scene(ctx, sc).build(accel, mode).trace_closest(axis)
        assert hits_equal(g, O.OrcScene(sc, oacc).trace_closest(axis)).all()
    g = Scene(ctx, sc).build(2, 0).trace_closest(axis)
    assert (~hits_equal(g, naive) & ~near_tie_mask(axis, g, naive)).sum() == 0


def test_host_and_device_buffers_agree(ctx):
    import torch
    sc = scenes.triangle_soup(5000, 1, 64, 64)
    rays = random_rays(5000, seed=8)
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH)
    host = g.trace_closest(rays)
    dev_rays = torch.from_numpy(rays.view(np.uint8).reshape(len(rays), 32)).cuda()
    dev_hits = g.trace_closest(dev_rays)
    torch.cuda.synchronize()
    got = dev_hits.cpu().numpy().view(np.uint32).reshape(-1, 2)
    assert (got[:, 1] == host["id"]).all() and (got[:, 0] == host["t"].view(np.uint32)).all()


@pytest.mark.slow
def test_soup_1080p_camera_rays(ctx):
    """1,000,000-triangle soup (seed 0), 1920x1080 camera rays (every 97th pixel): FAST BVH hit ids
    equal the exact closest hit; grid at G = 128 (the reference's rule) and at G = 100 (cbrt(N),
    with the reference's shift indexing) equal the restated grid bit for bit."""
    sc = scenes.triangle_soup(1_000_000, 0, 1920, 1080)
    rays = camera_rays(sc.camera, 1920, 1080, step=97)
    exact = O.OrcScene(sc, 3).trace_closest(rays)
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    gh = g.trace_closest(rays)
    ties = near_tie_mask(rays, gh, exact)
    bad = ~hits_equal(gh, exact) & ~ties
    assert not bad.any(), f"{bad.sum()} / {len(rays)} differ"
    assert (gh["id"] != capi.MRT_HIT_NONE).sum() > len(rays) // 4
    for G, index in ((0, capi.MRT_GRID_INDEX_REFERENCE), (100, capi.MRT_GRID_INDEX_REFERENCE),
                     (100, capi.MRT_GRID_INDEX_LINEAR)):
        gg = Scene(ctx, sc).build(capi.MRT_ACCEL_REGULAR_GRID, grid_size=G, grid_index=index)
        og = O.OrcScene(sc, 1, grid_size=G, grid_index=index)
        sub = rays[::4]
        assert hits_equal(gg.trace_closest(sub), og.trace_closest(sub)).all(), (G, index)


@pytest.mark.parametrize("grid_size,grid_index", [(0, capi.MRT_GRID_INDEX_REFERENCE), (37, capi.MRT_GRID_INDEX_LINEAR)])
def test_grid_counting_replay_equals_the_oracle_walk(ctx, grid_size, grid_index):
    """The grid's counting replay (cells visited, triangle references tested: the algorithmic bytes of
    the grid roofline) equals the oracle's count of the same walk, ray by ray."""
    sc = scenes.triangle_soup(20000, 3, 320, 240)
    rays = np.concatenate([random_rays(5000, seed=13), camera_rays(sc.camera, 320, 240, step=7)])
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_REGULAR_GRID, grid_size=grid_size, grid_index=grid_index)
    cells, refs = g.trace_counts(rays)
    o = O.OrcScene(sc, 1, grid_size=grid_size, grid_index=grid_index)
    oc, orf = o.grid_counts(rays)
    assert np.array_equal(cells, oc) and np.array_equal(refs, orf)
    assert cells.min() >= 1 and refs.sum() > len(rays)


def test_fast_counting_replay_bounds(ctx):
    """FAST BVH counting replay: a ray that misses the scene's box fetches the root node only; every
    ray that hits a triangle fetched at least one triangle record."""
    sc = scenes.triangle_soup(20000, 3, 320, 240)
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    rays = random_rays(4000, seed=17)
    miss = np.zeros(2, rays.dtype)
    miss["origin"] = [[5.0, 5.0, 5.0], [-5.0, 5.0, 5.0]]
    miss["direction"] = [[0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]
    miss["depth"] = 1
    miss["exclude"] = 0xFFFFFFFF
    rays = np.concatenate([rays, miss])
    nodes, tris = g.trace_counts(rays)
    hits = g.trace_closest(rays)
    assert (tris[-2:] == 0).all() and (nodes[-2:] <= 4).all()
    hit = (hits["id"] >> 30) == capi.MRT_PRIM_TRIANGLE
    assert hit.any() and (tris[hit] >= 1).all() and (nodes >= 1).all()
