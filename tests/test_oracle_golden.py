"""The oracle (C restatement) pinned to the reference: its own unit-test vectors, and outputs of the
reference's compiled code committed as golden fixtures (tests/golden/make_golden.py).  CPU only."""
import json
import os
import zlib

import numpy as np
import pytest

import orc as O
from helpers import random_rays
from mobileraytracer_b200 import capi, scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
UNIT = json.load(open(os.path.join(GOLDEN, "reference_unit_tests.json")))["cases"]
OUTPUTS = json.load(open(os.path.join(GOLDEN, "reference_outputs.json")))


def _ref_available():
    try:
        O.ref()
        return True
    except RuntimeError:
        return False


def _normalize32(v):
    v = np.asarray(v, np.float32)
    d = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]
    return v * (np.float32(1.0) / np.sqrt(np.float32(d)))


def _libs():
    libs = [("restatement", O.orc(), "orc_")]
    if _ref_available():
        libs.append(("reference", O.ref(), "ref_"))
    return libs


@pytest.mark.parametrize("case", UNIT, ids=lambda c: c["name"])
def test_reference_unit_vectors(case):
    """TestTriangle.cpp / TestPlane.cpp assertions, against the restatement and the compiled reference."""
    for who, lib, p in _libs():
        fn = lambda n: getattr(lib, p + n)
        kind = case["kind"]
        if kind == "triangle_box":
            abc = O.f32(*sum(case["triangle"], []))
            got = fn("triangle_intersect_box")(O.fptr(abc), O.fptr(O.f32(*case["min"])), O.fptr(O.f32(*case["max"])))
            assert bool(got) == case["expect"], who
        elif kind == "triangle_ray":
            abc = O.f32(*sum(case["triangle"], []))
            o = O.f32(*case["origin"])
            d = O.f32(*case["target"]) - o
            t = np.zeros(1, np.float32)
            got = fn("triangle_intersect")(O.fptr(abc), None, None, O.fptr(o), O.fptr(d), np.float32(1e30), O.fptr(t), None, None)
            assert bool(got) == case["expect"], who
        elif kind == "triangle_normal":
            abc = O.f32(*sum(case["triangle"], []))
            normals = np.concatenate([_normalize32(n) for n in case["normals_unnormalised"]]).astype(np.float32)
            colors = O.f32(*sum(case["colors"], []))
            t, n, c = np.zeros(1, np.float32), np.zeros(3, np.float32), np.zeros(3, np.float32)
            got = fn("triangle_intersect")(O.fptr(abc), O.fptr(normals), O.fptr(colors), O.fptr(O.f32(*case["origin"])),
                                          O.fptr(O.f32(*case["direction"])), np.float32(1e30), O.fptr(t), O.fptr(n), O.fptr(c))
            assert got == 1, who
            if case["expect_vertex"]:
                k = "ABC".index(case["expect_vertex"])
                assert (n == normals[3 * k:3 * k + 3]).all(), (who, n, normals[3 * k:3 * k + 3])
        elif kind == "triangle_aabb":
            if who == "reference":
                out = np.zeros(15, np.float32)
                lib.ref_triangle_fields(O.fptr(O.f32(*sum(case["triangle"], []))), O.fptr(out))
                assert (out[9:12] == case["min"]).all() and (out[12:15] == case["max"]).all()
        elif kind == "plane_box":
            pn = O.f32(*case["plane"]["point"], *case["plane"]["normal"])
            got = fn("plane_intersect_box")(O.fptr(pn), O.fptr(O.f32(*case["min"])), O.fptr(O.f32(*case["max"])))
            assert bool(got) == case["expect"], who
        elif kind == "plane_distance_at_least":
            pn = O.f32(*case["plane"]["point"], *case["plane"]["normal"])
            got = fn("plane_distance")(O.fptr(pn), O.fptr(O.f32(*case["point"])))
            assert case["expect_ge"] <= got, who


def test_reference_outputs_closest_hits():
    """Closest-hit ids and distance bits of the reference's compiled accelerators (golden)."""
    rays = random_rays(512, seed=OUTPUTS["rays_seed"])
    scs = {"glass_room": scenes.glass_room(), "cornell_box": scenes.cornell_box(),
           "soup2k": scenes.triangle_soup(2000, 7, 64, 64)}
    for key, want in OUTPUTS["closest"].items():
        name, accel = key.split("/")
        h = O.OrcScene(scs[name], int(accel)).trace_closest(rays)
        assert h["id"].tolist() == want["id"], key
        assert h["t"].view(np.uint32).tolist() == want["t_bits"], key


def test_reference_outputs_frames():
    """Whole NoShadows / Whitted frames of the reference Renderer (deterministic configuration)."""
    for key, crc in OUTPUTS["frames"].items():
        name, accel = key.split("/")
        sc = scenes.cornell_box() if name.startswith("cornell") else scenes.glass_room()
        sc.lights = [scenes.point_light((0.1, 0.45, -0.3))]
        shader = 0 if name.endswith("noshadows") else 1
        opts = capi.render_opts(shader=shader, width=64, height=64, spp=1, spl=1)
        bm, _, _ = O.OrcScene(sc, int(accel)).render(sc.camera, opts, threads=2)
        assert zlib.crc32(bm.tobytes()) == crc, key


@pytest.mark.skipif(not _ref_available(), reason="compiled reference not built (make -C oracle ref)")
@pytest.mark.parametrize("accel", [0, 1, 2])
def test_restatement_equals_reference_traces(accel):
    for sc in (scenes.glass_room(), scenes.cornell_box(), scenes.triangle_soup(8000, 4, 64, 64)):
        rays = random_rays(6000, seed=13)
        r = O.RefScene(sc, accel).trace_closest(rays)
        o = O.OrcScene(sc, accel).trace_closest(rays)
        assert (r["id"] == o["id"]).all() and (r["t"].view(np.uint32) == o["t"].view(np.uint32)).all()
        dist = np.full(len(rays), 0.5, np.float32)
        assert (O.RefScene(sc, accel).trace_any(rays, dist) == O.OrcScene(sc, accel).trace_any(rays, dist)).all()


@pytest.mark.skipif(not _ref_available(), reason="compiled reference not built (make -C oracle ref)")
def test_restatement_equals_reference_frames():
    """Deterministic shader configurations: one point light, Constant(0.5) sampler."""
    for sc, shader in ((scenes.glass_room(), 0), (scenes.glass_room(), 1), (scenes.cornell_box(), 1),
                       (scenes.triangle_soup(5000, 2, 96, 64), 0)):
        sc.lights = [scenes.point_light((0.1, 0.45, -0.3))]
        for accel in (0, 1, 2):
            opts = capi.render_opts(shader=shader, width=96, height=64, spp=1, spl=1)
            bm_r, _, _ = O.ref_render(sc, sc.camera, opts, accel, threads=4)
            bm_o, _, _ = O.OrcScene(sc, accel).render(sc.camera, opts, threads=4)
            assert (bm_r == bm_o).all()


@pytest.mark.skipif(not _ref_available(), reason="compiled reference not built (make -C oracle ref)")
def test_restatement_equals_reference_depthmap_diffuse_orthographic():
    """DepthMap and DiffuseMaterial frames, and every direct shader through an Orthographic camera
    (whose film rectangle also widens the grid bounds, Orthographic.cpp:36-46), on every accelerator."""
    ortho = scenes.orthographic((0.3, 0.2, -3.4), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 2.6, 1.9)
    for sc in (scenes.glass_room(), scenes.cornell_box(), scenes.triangle_soup(5000, 2, 96, 64)):
        sc.lights = [scenes.point_light((0.1, 0.45, -0.3))]
        for cam in (sc.camera, ortho):
            for shader in (0, 3, 4):
                for accel in (0, 1, 2):
                    if shader == 0 and cam is sc.camera:
                        continue   # covered above
                    opts = capi.render_opts(shader=shader, width=96, height=64, spp=1, spl=1,
                                            depth_point=(1.5, 1.0, 2.0))
                    sc.camera = cam
                    bm_r, _, _ = O.ref_render(sc, cam, opts, accel, threads=4)
                    bm_o, _, _ = O.OrcScene(sc, accel).render(cam, opts, threads=4)
                    assert (bm_r == bm_o).all(), (shader, accel, cam.kind)
                    assert np.count_nonzero(bm_o & 0xFFFFFF) > 20


@pytest.mark.skipif(not _ref_available(), reason="compiled reference not built (make -C oracle ref)")
def test_restatement_scalar_functions():
    ref, orc = O.ref(), O.orc()
    for i in range(300):
        for b in (2, 3, 5, 7):
            assert ref.ref_halton(i, b) == orc.orc_halton(i, b)
    u = scenes.uniform(5, 4000).reshape(-1, 4)
    for k in range(len(u)):
        rgb = O.f32(u[k, 0] * 3 - 0.5, u[k, 1] * 1.2, u[k, 2] * 300)
        avg = int(u[k, 3] * 0xFFFFFFFF)
        n = 1 + (k % 70)
        assert ref.ref_incremental_avg(O.fptr(rgb), avg, n) == orc.orc_incremental_avg(O.fptr(rgb), avg, n)
    cams = [scenes.cornell_box().camera, scenes.cli_camera(1920, 1080), scenes.heightfield(4).camera]
    a, b = np.zeros(6, np.float32), np.zeros(6, np.float32)
    for cam in cams:
        for k in range(200):
            uv = (float(u[k, 0]), float(u[k, 1]), float(u[k, 2] * 1e-3), float(u[k, 3] * -1e-3))
            ref.ref_camera_ray(__import__("ctypes").byref(cam), *uv, O.fptr(a))
            orc.orc_camera_ray(__import__("ctypes").byref(cam), *uv, O.fptr(b))
            assert (a == b).all()
