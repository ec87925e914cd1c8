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


# ---- the conversion pinned to the reference's own OBJLoader::fillScene ----------------------------
# OBJLoader::fillScene (OBJLoader.cpp:68-248), compiled from the reference sources, runs on the
# oracle's restatement of tinyobjloader's parse (the library is an absent submodule); its Scene must
# equal the library loader's output bit for bit.  A face vertex without a normal in a file that has
# normals makes the reference read normals[-1] (OBJLoader.cpp:111-124, undefined behaviour), so these
# fixtures give either every face vertex a normal or the file none.

def _write_random_obj(path_obj, path_mtl, seed: int, with_normals: bool):
    rng = np.random.default_rng(seed)
    mtl = ["newmtl white", "Kd 0.73 0.73 0.73",
           "newmtl white_close", "Kd 0.7300004 0.73 0.73",       # within Epsilon of white: merged
           "newmtl white_far", "Kd 0.7300100 0.73 0.73",         # not merged
           "newmtl mirror", "Kd 0 0 0", "Ks 1.7 1.6 1.5",
           "newmtl glass", "Tf 0.9 0.8 0.7", "d 0.25", "Ni 1.45",
           "newmtl frosted", "Kd 0.2 0.3 0.4", "Kt 0.8 0.8 0.8", "Tr 0.6", "Ni 1.2",
           "newmtl lamp", "Ke 12 9 3",
           "newmtl dim", "Ke 0.4 0.9 0.2",
           "newmtl lamp_close", "Ke 12.000001 9 3"]
    open(path_mtl, "w").write("\n".join(mtl) + "\n")
    names = ["white", "white_close", "white_far", "mirror", "glass", "frosted", "lamp", "dim", "lamp_close",
             "not_defined"]
    lines = ["# generated fixture"]
    nv = 0
    nn = 0
    for f in range(120):
        if f % 7 == 0:
            lines.append(f"usemtl {names[int(rng.integers(len(names)))]}")
        k = int(rng.choice([3, 3, 3, 4, 5]))
        for _ in range(k):
            p = rng.uniform(-1, 1, 3)
            if rng.random() < 0.5:
                c = rng.uniform(0, 1, 3)
                lines.append("v %.7g %.7g %.7g %.5g %.5g %.5g" % (*p, *c))
            else:
                lines.append("v %.7g %.7g %.7g" % tuple(p))
            nv += 1
            if with_normals:
                q = rng.normal(size=3) * (1.0 if rng.random() < 0.9 else 0.0)   # some zero normals
                lines.append("vn %.6g %.6g %.6g" % tuple(q))
                nn += 1
        toks = []
        for j in range(k):
            vi = nv - k + 1 + j
            v = str(vi) if rng.random() < 0.5 else str(vi - nv - 1)      # absolute or relative
            if with_normals:
                ni = nn - k + 1 + j
                toks.append(f"{v}//{ni}")
            else:
                toks.append(v)
        lines.append("f " + " ".join(toks))
    open(path_obj, "w").write("\n".join(lines) + "\n")


def _check_against_reference_fill(obj, mtl):
    import orc as O
    parsed = obj_oracle.parse(obj, mtl)
    tri, mats, lights = O.ref_obj_fill(obj, mtl, parsed)
    s = scenes.load_obj(obj, mtl)
    F = np.float32
    n = s.n_triangles
    assert len(tri) == n and len(mats) == len(s.materials) and len(lights) == len(s.lights)
    A = s.tri_abc[:, 0:3]
    want = np.concatenate([A, s.tri_abc[:, 3:6] - A, s.tri_abc[:, 6:9] - A, s.tri_normals, s.tri_colors], 1).astype(F)
    assert np.array_equal(tri[:, :27].view(np.uint32), want.view(np.uint32))
    assert np.array_equal(tri[:, 27].view(np.int32), s.tri_material)
    got_m = np.array([[*m.le, *m.kd, *m.ks, *m.kt, m.ior] for m in s.materials], F).reshape(-1, 13)
    assert np.array_equal(mats.view(np.uint32), got_m.view(np.uint32))
    got_l = np.array([[*l.p0, *(np.array(l.p1, F) - np.array(l.p0, F)), *(np.array(l.p2, F) - np.array(l.p0, F)),
                       *l.radiance.le, *l.radiance.kd, *l.radiance.ks, *l.radiance.kt, l.radiance.ior]
                      for l in s.lights], F).reshape(-1, 22)
    assert np.array_equal(lights.view(np.uint32), got_l.view(np.uint32))
    return n, len(mats), len(lights)


def test_room_without_normals_equals_reference_fill_scene(tmp_path):
    text = open(OBJ).read().splitlines()
    kept = []
    for line in text:
        if line.startswith("vn "):
            continue
        if line.startswith("f "):
            line = "f " + " ".join(t.split("/")[0] for t in line.split()[1:])
        kept.append(line)
    obj = str(tmp_path / "room_plain.obj")
    open(obj, "w").write("\n".join(kept) + "\n")
    n, m, l = _check_against_reference_fill(obj, MTL)
    assert (n, l) == (17, 3) and m == 5


@pytest.mark.parametrize("seed,with_normals", [(1, True), (2, False), (3, True)])
def test_generated_scenes_equal_reference_fill_scene(tmp_path, seed, with_normals):
    obj, mtl = str(tmp_path / "g.obj"), str(tmp_path / "g.mtl")
    _write_random_obj(obj, mtl, seed, with_normals)
    n, m, l = _check_against_reference_fill(obj, mtl)
    assert n > 0 and l > 0 and m > 0
