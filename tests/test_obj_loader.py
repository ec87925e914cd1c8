"""The library's OBJ / MTL loader (mrt_obj_load, host code) against the restatement of the
reference loader in oracle/obj_oracle.py, on a fixture that exercises every branch of
OBJLoader::fillScene (OBJLoader.cpp:68-248).  No GPU needed."""
import os

import numpy as np
import pytest

import obj_oracle
from mobileraytracer_b200 import MrtError, capi, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
OBJ = os.path.join(HERE, "golden", "obj", "room.obj")
MTL = os.path.join(HERE, "golden", "obj", "room.mtl")


def _mat_tuple(m):
    F = np.float32
    return (np.array(m.kd, F), np.array(m.ks, F), np.array(m.kt, F), F(m.ior), np.array(m.le, F))


def test_loader_equals_restatement():
    s = scenes.load_obj(OBJ, MTL)
    abc, nrm, col, mat, mats, lights = obj_oracle.load(OBJ, MTL)
    assert s.tri_abc.shape == abc.shape
    for got, want in ((s.tri_abc, abc), (s.tri_normals, nrm), (s.tri_colors, col)):
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(s.tri_material, mat)
    assert len(s.materials) == len(mats)
    for m, w in zip(s.materials, mats):
        for a, b in zip(_mat_tuple(m), w):
            assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))
    assert len(s.lights) == len(lights)
    for l, (a, b, c, m) in zip(s.lights, lights):
        assert l.kind == capi.MRT_LIGHT_AREA
        for got, want in ((l.p0, a), (l.p1, b), (l.p2, c)):
            assert np.array_equal(np.array(got, np.float32), want)
        for x, y in zip(_mat_tuple(l.radiance), m):
            assert np.array_equal(np.asarray(x), np.asarray(y, np.float32))


def test_loader_conventions():
    """The fixture's expected structure, stated by hand from OBJLoader.cpp."""
    s = scenes.load_obj(OBJ, MTL)
    # 5 walls x 2 + 3 prop triangles + pentagon fan (3) + the mixed-normal face; lamp quad (2) and
    # the dim lamp (1) are lights
    assert s.n_triangles == 10 + 3 + 3 + 1 and len(s.lights) == 3
    assert len(s.materials) == 5                          # white_again merged into white
    assert list(s.tri_material[:2]) == [-1, -1]           # before any usemtl
    assert list(s.tri_material[2:6]) == [0, 0, 0, 0]      # white, white_again
    assert list(s.tri_material[8:10]) == [-1, -1]         # unknown material name
    assert abs(s.materials[2].ks[0] - 0.9) < 1e-6         # mirror: Ks / 2
    assert abs(s.materials[3].kt[0] - 0.9) < 1e-6         # glass: Tf * (1 - d)
    assert abs(s.materials[4].kt[0] - 0.8 * 0.25) < 1e-6  # frosted: Kt * (1 - (1 - Tr))
    assert s.lights[0].radiance.le[0] == 1.0 and abs(s.lights[0].radiance.le[1] - 0.8) < 1e-6   # Ke / max
    assert s.lights[2].radiance.le[0] == 0.5                                                    # not scaled
    assert s.tri_abc[0, 0] == 1.0                        # x negated: vertex 1 (-1, -1, -1)
    assert np.allclose(s.tri_normals[2, :3], [0.0, -1.0, 0.0])   # given normal, normalised
    assert np.allclose(s.tri_colors[10, :3], [0.9, 0.1, 0.1])    # vertex colour


def test_loader_errors(tmp_path):
    with pytest.raises(MrtError) as e:
        scenes.load_obj(str(tmp_path / "missing.obj"))
    assert e.value.status == capi.MRT_ERR_ARG and "cannot open" in str(e.value)
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nf 1 2 7\n")
    with pytest.raises(MrtError) as e:
        scenes.load_obj(str(bad))
    assert "face index" in str(e.value)
    s = scenes.load_obj(OBJ)       # no MTL: every face without material, no lights
    assert len(s.lights) == 0 and (s.tri_material == -1).all() and s.n_triangles == 10 + 3 + 3 + 2 + 1 + 1
