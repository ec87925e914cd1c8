"""Edge cases of the scene contents on the device (GPU), each against the oracle: no triangles,
one triangle (a tree that is a single leaf), no lights, only planes and spheres, rays that miss
everything, and the same through the batch and the whole-path launches."""
import numpy as np
import pytest

import orc as O
from mobileraytracer_b200 import Batch, Scene, capi, scenes

pytestmark = pytest.mark.gpu

NS, WH, PT = capi.MRT_SHADER_NOSHADOWS, capi.MRT_SHADER_WHITTED, capi.MRT_SHADER_PATHTRACER


def _variants():
    gr = scenes.glass_room()
    no_tri = scenes.glass_room()
    no_tri.tri_abc = np.zeros((0, 9), np.float32)
    no_tri.tri_normals = None
    no_tri.tri_colors = None
    no_tri.tri_material = np.zeros(0, np.int32)
    one_tri = scenes.glass_room()
    one_tri.tri_abc = gr.tri_abc[:1].copy()
    one_tri.tri_normals = gr.tri_normals[:1].copy()
    one_tri.tri_colors = gr.tri_colors[:1].copy()
    one_tri.tri_material = gr.tri_material[:1].copy()
    no_light = scenes.glass_room()
    no_light.lights = []
    empty = scenes.Scene()
    empty.camera = gr.camera
    return {"no_triangles": no_tri, "one_triangle": one_tri, "no_lights": no_light, "empty": empty}


@pytest.mark.parametrize("name", ["no_triangles", "one_triangle", "no_lights", "empty"])
@pytest.mark.parametrize("shader", [NS, WH, PT])
def test_edge_scene(ctx, name, shader):
    torch = pytest.importorskip("torch")
    sc = _variants()[name]
    opts = capi.render_opts(shader=shader, width=48, height=32, spp=2, spl=2, seed=4)
    for accel, mode, oacc in ((capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, 3), (capi.MRT_ACCEL_REGULAR_GRID, 0, 1),
                              (capi.MRT_ACCEL_BVH, capi.MRT_BVH_REFERENCE, 2)):
        g = Scene(ctx, sc).build(accel, mode, camera=sc.camera)
        bm_g, acc_g, st = g.render(sc.camera, opts, accum=np.zeros((32, 48, 4), np.float32))
        bm_o, acc_o, counts = O.OrcScene(sc, oacc, camera=sc.camera).render(sc.camera, opts)
        assert np.array_equal(bm_g, bm_o), (name, accel, mode)
        assert (st.rays_closest, st.rays_shadow) == tuple(counts[:2])
        if accel == capi.MRT_ACCEL_BVH and mode == capi.MRT_BVH_FAST:
            b = Batch(ctx, wave_roots=1024, pipelines=1, block_threads=128, blocks_per_sm=8, max_spl=2)
            bm = torch.zeros((32, 48), dtype=torch.int32, device="cuda")
            b.submit(g, sc.camera, opts, bm)
            b.run()
            b.close()
            assert np.array_equal(bm.cpu().numpy().view(np.uint32), bm_o)
    if name == "empty":
        assert not (bm_g & 0xFFFFFF).any()


def test_rays_that_miss_everything(ctx):
    sc = scenes.cornell_box()
    g = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST)
    rays = np.zeros(1000, [("origin", np.float32, 3), ("direction", np.float32, 3), ("depth", np.int32),
                           ("exclude", np.uint32)])
    rays["origin"] = (0.0, 0.0, -5.0)
    rays["direction"] = (0.0, 0.0, -1.0)     # away from the box
    rays["exclude"] = 0xFFFFFFFF
    hits = g.trace_closest(rays)
    assert (hits["id"] == capi.MRT_HIT_NONE).all() and (hits["t"] == np.float32(1e30)).all()
    occ = g.trace_any(rays, np.full(1000, 100.0, np.float32))
    assert not occ.any()
