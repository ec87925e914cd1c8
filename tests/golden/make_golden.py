"""Regenerates the golden fixtures in this directory from the reference checkout.

    python tests/golden/make_golden.py [/path/to/MobileRayTracer]

reference_unit_tests.json: the input/expected pairs of the reference's own gtest cases for the
render path, read from app/Unit_Testing/TestTriangle.cpp and TestPlane.cpp (parsed as text: the
fixture triangle/plane, the boxes, the rays and the asserted booleans).

reference_outputs.json: outputs of the reference's own compiled code (oracle/_ref/liboracle_ref.so,
built by `make -C oracle ref`) on small seeded inputs: closest-hit ids and distance bits of 512 rays
in three scenes for each accelerator, and CRC32s of whole NoShadows / Whitted frames rendered by the
reference Renderer in configurations where it is deterministic (one point light, Constant(0.5)).
"""
from __future__ import annotations

import json
import os
import re
import sys
import zlib

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

NUM = r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?f?"


def vec(text):
    return [float(x.rstrip("f")) for x in re.findall(NUM, text)]


def parse_triangle_tests(src: str):
    cases = []
    fixture = [[0, 0, 0], [0, 1, 0], [0, 0, 1]]
    for m in re.finditer(r"TEST_F\(TestTriangle,\s*(\w+)\)\s*\{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(2)
        tri = fixture
        t2 = re.search(r"Triangle\s+\w+\s*\{\s*::glm::vec3\s*\{([^}]*)\},\s*::glm::vec3\s*\{([^}]*)\},\s*::glm::vec3\s*\{([^}]*)\}", body)
        if t2:
            tri = [vec(t2.group(1)), vec(t2.group(2)), vec(t2.group(3))]
        expect = re.search(r"ASSERT_EQ\((true|false),\s*intersected\)", body)
        if name.startswith("intersectBox"):
            mn = re.search(r"min\s*\{([^}]*)\}", body)
            mx = re.search(r"max\s*\{([^}]*)\}", body)
            cases.append({"kind": "triangle_box", "name": name, "triangle": tri, "min": vec(mn.group(1)),
                          "max": vec(mx.group(1)), "expect": expect.group(1) == "true"})
        elif name.startswith("intersectRay"):
            orig = re.search(r"orig\s*\{([^}]*)\}", body)
            target = re.search(r"dir\s*\{::glm::vec3\s*\{([^}]*)\}\s*-\s*orig\}", body)
            cases.append({"kind": "triangle_ray", "name": name, "triangle": tri, "origin": vec(orig.group(1)),
                          "target": vec(target.group(1)), "expect": expect.group(1) == "true"})
        elif name.startswith("normalTest"):
            orig = re.search(r"orig\s*\{([^}]*)\}", body)
            d = re.search(r"dir\s*\{([^}]*)\}", body)
            normals = re.findall(r"::glm::normalize\(::glm::vec3\{([^}]*)\}\)", body)
            colors = re.findall(r"::glm::vec3\{([^}]*)\}\}?\)?;?", body.split("normalize")[-1])
            which = re.search(r"triangle2\.normal([ABC])_", body)
            cases.append({"kind": "triangle_normal", "name": name, "triangle": tri, "origin": vec(orig.group(1)),
                          "direction": vec(d.group(1)), "normals_unnormalised": [vec(n) for n in normals],
                          "colors": [[1, 0, 0], [0, 1, 0], [0, 0, 1]],
                          "expect_vertex": which.group(1) if which else None})
        elif name == "AABB":
            mins = re.findall(r"ASSERT_EQ\(([-\d.f]+),\s*box\.pointMin_\[(\d)\]\)", body)
            maxs = re.findall(r"ASSERT_EQ\(([-\d.f]+),\s*box\.pointMax_\[(\d)\]\)", body)
            cases.append({"kind": "triangle_aabb", "name": name, "triangle": tri,
                          "min": [float(v.rstrip("f")) for v, _ in sorted(mins, key=lambda x: x[1])],
                          "max": [float(v.rstrip("f")) for v, _ in sorted(maxs, key=lambda x: x[1])]})
    return cases


def parse_plane_tests(src: str):
    cases = []
    fixture = {"point": [-1, 0, 0], "normal": [1, 0, 0]}
    for m in re.finditer(r"TEST_F\(TestPlane,\s*(\w+)\)\s*\{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(2)
        plane = fixture
        p = re.search(r"Plane\s+plane\s*\{::glm::vec3\s*\{([^}]*)\},\s*::glm::vec3\s*\{([^}]*)\}", body)
        if p:
            plane = {"point": vec(p.group(1)), "normal": vec(p.group(2))}
        if "intersectBox" in body:
            b = re.search(r"AABB box\s*\{::glm::vec3\s*\{([^}]*)\},\s*::glm::vec3\s*\{([^}]*)\}\}", body)
            e = re.search(r"ASSERT_EQ\((true|false),\s*result\)", body)
            cases.append({"kind": "plane_box", "name": name, "plane": plane, "min": vec(b.group(1)),
                          "max": vec(b.group(2)), "expect": e.group(1) == "true"})
        elif "distance" in body:
            q = re.search(r"vec3 p\s*\{([^}]*)\}", body)
            e = re.search(r"expected\s*\{([^}]*)\}", body)
            cases.append({"kind": "plane_distance_at_least", "name": name, "plane": plane, "point": vec(q.group(1)),
                          "expect_ge": vec(e.group(1))[0]})
    return cases


def reference_outputs():
    import numpy as np

    import orc as O
    from helpers import random_rays
    from mobileraytracer_b200 import capi, scenes
    out = {"closest": {}, "frames": {}}
    scs = {"glass_room": scenes.glass_room(), "cornell_box": scenes.cornell_box(),
           "soup2k": scenes.triangle_soup(2000, 7, 64, 64)}
    rays = random_rays(512, seed=21)
    out["rays_seed"] = 21
    for name, sc in scs.items():
        for accel in (0, 1, 2):
            h = O.RefScene(sc, accel).trace_closest(rays, threads=1)
            out["closest"][f"{name}/{accel}"] = {"id": h["id"].tolist(), "t_bits": h["t"].view(np.uint32).tolist()}
    for name, sc, shader in (("glass_room_noshadows", scenes.glass_room(), 0), ("glass_room_whitted", scenes.glass_room(), 1),
                             ("cornell_whitted", scenes.cornell_box(), 1)):
        sc.lights = [scenes.point_light((0.1, 0.45, -0.3))]
        for accel in (0, 1, 2):
            opts = capi.render_opts(shader=shader, width=64, height=64, spp=1, spl=1)
            bm, _, _ = O.ref_render(sc, sc.camera, opts, accel, threads=1)
            out["frames"][f"{name}/{accel}"] = zlib.crc32(bm.tobytes())
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MRT_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout>  (or set MRT_REFERENCE_DIR)")
    tt = open(os.path.join(ref, "app/Unit_Testing/TestTriangle.cpp")).read()
    tp = open(os.path.join(ref, "app/Unit_Testing/TestPlane.cpp")).read()
    cases = parse_triangle_tests(tt) + parse_plane_tests(tp)
    json.dump({"source": "app/Unit_Testing/TestTriangle.cpp, app/Unit_Testing/TestPlane.cpp", "cases": cases},
              open(os.path.join(HERE, "reference_unit_tests.json"), "w"), indent=1)
    print(f"{len(cases)} unit-test cases")
    json.dump(reference_outputs(), open(os.path.join(HERE, "reference_outputs.json"), "w"))
    print("reference outputs written")


if __name__ == "__main__":
    main()
