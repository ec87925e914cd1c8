"""A scene read from OBJ / MTL (mrt_obj_load) rendered on the device against the oracle (GPU):
given and computed normals, vertex colours, mirror, glass and frosted materials, emitting faces as
area lights."""
import os

import numpy as np
import pytest

import orc as O
from mobileraytracer_b200 import Scene, capi, scenes

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("shader", [capi.MRT_SHADER_WHITTED, capi.MRT_SHADER_PATHTRACER, capi.MRT_SHADER_DIFFUSE])
@pytest.mark.parametrize("accel,mode,oacc", [(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, 3),
                                             (capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST, 1)])
def test_obj_scene_render(ctx, shader, accel, mode, oacc):
    cam = scenes.camera((0.0, 0.1, -2.6), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 55.0, 55.0)
    sc = scenes.load_obj(os.path.join(HERE, "golden", "obj", "room.obj"),
                         os.path.join(HERE, "golden", "obj", "room.mtl"), camera=cam)
    opts = capi.render_opts(shader=shader, width=80, height=64, spp=3, spl=2, seed=12, depth_min=2, depth_max=6)
    g = Scene(ctx, sc).build(accel, mode, camera=cam)
    bm_g, acc_g, stats = g.render(cam, opts, accum=np.zeros((64, 80, 4), np.float32))
    bm_o, acc_o, counts = O.OrcScene(sc, oacc, camera=cam).render(cam, opts)
    assert int(np.sum(bm_g != bm_o)) == 0
    assert float(np.abs(acc_g[..., :3] - acc_o[..., :3]).max()) <= (1e-3 if shader == capi.MRT_SHADER_PATHTRACER else 1e-4)
    assert (stats.rays_closest, stats.rays_shadow) == tuple(counts[:2])
    assert np.count_nonzero(bm_g & 0xFFFFFF) > 2000
