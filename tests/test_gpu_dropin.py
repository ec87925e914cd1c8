"""The C++ drop-in (reference class names and constructors over the C ABI): a reference-style client
program builds the scene through MobileRT::Scene / Components::* and calls Renderer::renderFrame;
its bitmap must equal the C ABI's render of the same arrays (itself parity-checked against the
oracle).  The program is compiled here with g++ against cpp/include and libmrt_dropin.so."""
import os
import struct
import subprocess

import numpy as np
import pytest

from mobileraytracer_b200 import Scene, capi, scenes
from mobileraytracer_b200.build import DROPIN_OUT, HERE, build_dropin

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _write_scene(path, sc, opts, accel, bvh_mode):
    f = open(path, "wb")
    pack = lambda fmt, *v: f.write(struct.pack("<" + fmt, *v))
    n = sc.n_triangles
    has_n, has_c = sc.tri_normals is not None, sc.tri_colors is not None
    pack("III", n, int(has_n), int(has_c))
    for i in range(n):
        f.write(sc.tri_abc[i].astype("<f4").tobytes())
        if has_n:
            f.write(sc.tri_normals[i].astype("<f4").tobytes())
        if has_c:
            f.write(sc.tri_colors[i].astype("<f4").tobytes())
        pack("i", int(sc.tri_material[i]))
    pack("I", len(sc.spheres))
    for i in range(len(sc.spheres)):
        f.write(sc.spheres[i].astype("<f4").tobytes())
        pack("i", int(sc.sphere_material[i]))
    pack("I", len(sc.planes))
    for i in range(len(sc.planes)):
        f.write(sc.planes[i].astype("<f4").tobytes())
        pack("i", int(sc.plane_material[i]))

    def mat(m):
        pack("13f", *m.le, *m.kd, *m.ks, *m.kt, m.ior)

    pack("I", len(sc.materials))
    for m in sc.materials:
        mat(m)
    pack("I", len(sc.lights))
    for l in sc.lights:
        pack("i", l.kind)
        pack("9f", *l.p0, *l.p1, *l.p2)
        mat(l.radiance)
    c = sc.camera
    pack("11f", *c.position, *c.look_at, *c.up, c.fov_h_deg, c.fov_v_deg)
    pack("iiiIIIIifii", opts.shader, accel, bvh_mode, opts.width, opts.height, opts.spp, opts.spl, opts.pixel_sampler,
         opts.constant_value, opts.light_sampler, opts.rr_sampler)
    f.close()


@pytest.fixture(scope="module")
def client(tmp_path_factory):
    build_dropin()
    exe = str(tmp_path_factory.mktemp("dropin") / "dropin_render")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-I", os.path.join(HERE, "cpp", "include"), "-I",
                    os.path.join(HERE, "cpp", "glm_min"), os.path.join(ROOT, "tests", "cpp", "dropin_render.cpp"),
                    "-L", os.path.dirname(DROPIN_OUT), "-lmrt_dropin", "-lmrt_cuda",
                    "-Wl,-rpath," + os.path.dirname(DROPIN_OUT), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("shader,accel,mode", [
    (capi.MRT_SHADER_NOSHADOWS, capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST),
    (capi.MRT_SHADER_WHITTED, capi.MRT_ACCEL_BVH, capi.MRT_BVH_REFERENCE),
    (capi.MRT_SHADER_WHITTED, capi.MRT_ACCEL_REGULAR_GRID, capi.MRT_BVH_FAST),
    (capi.MRT_SHADER_PATHTRACER, capi.MRT_ACCEL_NAIVE, capi.MRT_BVH_FAST),
])
def test_renderframe_through_the_dropin(ctx, client, tmp_path, shader, accel, mode):
    for sc in (scenes.glass_room(), scenes.cornell_box()):
        opts = capi.render_opts(shader=shader, width=80, height=48, spp=2, spl=1)
        path, out, pv = str(tmp_path / "scene.bin"), str(tmp_path / "out.bin"), str(tmp_path / "preview.bin")
        _write_scene(path, sc, opts, accel, mode)
        r = subprocess.run([client, path, out, pv], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = np.fromfile(out, np.uint32).reshape(48, 80)
        g = Scene(ctx, sc).build(accel, mode)
        want, _, _ = g.render(sc.camera, opts)
        assert (got == want).all()
        # Renderer::rasterPreview (the front end's first image) equals the C ABI's preview
        want_pv, _ = g.raster_preview(sc.camera, 80, 48)
        assert (np.fromfile(pv, np.uint32).reshape(48, 80) == want_pv).all()


@pytest.fixture(scope="module")
def obj_client(tmp_path_factory):
    build_dropin()
    exe = str(tmp_path_factory.mktemp("dropin_obj") / "dropin_obj")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-I", os.path.join(HERE, "cpp", "include"), "-I",
                    os.path.join(HERE, "cpp", "glm_min"), os.path.join(ROOT, "tests", "cpp", "dropin_obj.cpp"),
                    "-L", os.path.dirname(DROPIN_OUT), "-lmrt_dropin", "-lmrt_cuda",
                    "-Wl,-rpath," + os.path.dirname(DROPIN_OUT), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("shader,ortho", [(capi.MRT_SHADER_WHITTED, 0), (capi.MRT_SHADER_DEPTHMAP, 1),
                                          (capi.MRT_SHADER_DIFFUSE, 0)])
def test_obj_scene_through_the_dropin(ctx, obj_client, tmp_path, shader, ortho):
    """Components::OBJLoader + DepthMap / DiffuseMaterial / Orthographic through the drop-in: equal to
    the C ABI render of the scene mrt_obj_load reads."""
    obj = os.path.join(ROOT, "tests", "golden", "obj", "room.obj")
    mtl = os.path.join(ROOT, "tests", "golden", "obj", "room.mtl")
    out = str(tmp_path / "out.bin")
    r = subprocess.run([obj_client, obj, mtl, str(shader), str(ortho), "64", "48", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.uint32).reshape(48, 64)
    if ortho:
        cam = scenes.orthographic((0.0, 0.1, -2.6), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 2.4, 2.0)
    else:
        cam = scenes.camera((0.0, 0.1, -2.6), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 55.0, 55.0)
    sc = scenes.load_obj(obj, mtl, camera=cam)
    opts = capi.render_opts(shader=shader, width=64, height=48, spp=1, spl=1, depth_point=(1.5, 1.0, 2.0))
    want, _, _ = Scene(ctx, sc).build(capi.MRT_ACCEL_BVH, capi.MRT_BVH_FAST, camera=cam).render(cam, opts)
    assert (got == want).all()
    assert np.count_nonzero(want & 0xFFFFFF) > 500
