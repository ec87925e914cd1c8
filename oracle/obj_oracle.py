"""Restatement of the reference OBJ loader for the tests (TEST INFRASTRUCTURE ONLY).

OBJLoader::process + OBJLoader::fillScene (app/Components/ObjectLoaders/OBJLoader.cpp:21-248) over
tinyobjloader's LoadObj with triangulation on (OBJLoader.cpp:33-35).  tinyobjloader is an empty,
unpinned submodule in the reference checkout, so neither it nor the loader can be compiled here:
this file restates both from their published behaviour and from OBJLoader.cpp as read, independently
of the library's C++ loader, and the tests compare the two.  The conversion step is also pinned to
the reference's own code: parse() feeds OBJLoader::fillScene, compiled from the reference sources
(oracle/ref_driver.cpp, ref_obj_fill), and the tests compare its Scene with the library's loader.
Only the parsing (tinyobjloader's, absent and unpinned) remains a restatement.

Float32 arithmetic with numpy follows the reference's operation order (glm: normalize =
v * (1 / sqrt(dot)), dot = (x*x + y*y) + z*z, cross as in the GLSL definition).
"""
from __future__ import annotations

import numpy as np

F = np.float32
EPS = F(1.0e-6)   # Utils.hpp:37


def _num(tok: str) -> F:
    return F(float(tok))


def _dot(a, b):
    return F(F(F(a[0] * b[0]) + F(a[1] * b[1])) + F(a[2] * b[2]))


def _normalize(v):
    inv = F(F(1.0) / np.sqrt(_dot(v, v)))
    return np.array([v[0] * inv, v[1] * inv, v[2] * inv], F)


def _cross(a, b):
    return np.array([F(a[1] * b[2]) - F(b[1] * a[2]), F(a[2] * b[0]) - F(b[2] * a[0]),
                     F(a[0] * b[1]) - F(b[0] * a[1])], F)


def read_mtl(path):
    """tinyobj material_t fields the loader reads, defaults of tinyobj's InitMaterial."""
    mats, names, cur = [], {}, None
    for raw in open(path):
        line = raw.split("#", 1)[0].split()
        if not line:
            continue
        key, args = line[0], line[1:]
        if key == "newmtl":
            cur = {"Kd": [F(0)] * 3, "Ks": [F(0)] * 3, "Kt": [F(0)] * 3, "Ke": [F(0)] * 3, "Ni": F(1), "d": F(1)}
            names[args[0]] = len(mats)
            mats.append(cur)
        elif cur is None:
            continue
        elif key in ("Kd", "Ks", "Kt", "Tf", "Ke") and args:
            v = [_num(a) for a in args[:3]]
            if len(v) < 3:
                v = [v[0]] * 3
            cur["Kt" if key == "Tf" else key] = v
        elif key == "d" and args:
            cur["d"] = _num(args[0])
        elif key == "Tr" and args:
            cur["d"] = F(F(1.0) - _num(args[0]))
        elif key == "Ni" and args:
            cur["Ni"] = _num(args[0])
    return mats, names


def _index(tok: str, n: int) -> int:
    i = int(tok)
    return i - 1 if i > 0 else n + i


def parse(obj_path, mtl_path=None):
    """tinyobjloader's LoadObj with triangulation, restated: (positions, vertex colours, normals,
    triangles as ((v, n), (v, n), (v, n), material), materials from read_mtl)."""
    mats, names = read_mtl(mtl_path) if mtl_path else ([], {})
    pos, col, nrm, tris = [], [], [], []
    cur = -1
    for raw in open(obj_path):
        line = raw.split("#", 1)[0].split()
        if not line:
            continue
        key, args = line[0], line[1:]
        if key == "v":
            v = [_num(a) for a in args]
            pos.append(v[:3])
            col.append(v[3:6] if len(v) >= 6 else [F(1), F(1), F(1)])
        elif key == "vn":
            nrm.append([_num(a) for a in args[:3]])
        elif key == "usemtl":
            cur = names.get(args[0], -1)
        elif key == "f":
            face = []
            for tok in args:
                parts = tok.split("/")
                vi = _index(parts[0], len(pos))
                ni = _index(parts[2], len(nrm)) if len(parts) >= 3 and parts[2] else -1
                face.append((vi, ni))
            for k in range(1, len(face) - 1):   # tinyobj triangulation: a fan from the first vertex
                tris.append((face[0], face[k], face[k + 1], cur))
    return pos, col, nrm, tris, mats


def load(obj_path, mtl_path=None):
    """(tri_abc, tri_normals, tri_colors, tri_material, materials, lights) as the reference builds
    the Scene; materials as (Kd, Ks, Kt, ior, Le) tuples, lights as (A, B, C, material)."""
    pos, col, nrm, tris, mats = parse(obj_path, mtl_path)
    abc, normals, colors, tmat, materials, lights = [], [], [], [], [], []
    for a, b, c, m in tris:
        p = [np.array([-pos[v][0], pos[v][1], pos[v][2]], F) for v, _ in (a, b, c)]
        cc = [np.array(col[v], F) for v, _ in (a, b, c)]
        n = []
        for _, ni in (a, b, c):
            if nrm and ni >= 0:
                q = nrm[ni]
                with np.errstate(all="ignore"):
                    n.append(_normalize(np.array([-q[0], q[1], q[2]], F)))
            else:
                n.append(np.zeros(3, F))
        has_normal = all(np.sqrt(_dot(x, x)) > 0 for x in n)
        mat_index = -1
        if m >= 0:
            t = mats[m]
            kd = np.array(t["Kd"], F)
            ks = np.array([x / F(2.0) for x in t["Ks"]], F)
            kt = np.array([x * F(F(1.0) - t["d"]) for x in t["Kt"]], F)
            e = [F(x) for x in t["Ke"]]
            mx = max(max(e[0], e[1]), e[2])
            if mx > F(1.0):
                e = [F(x / mx) for x in e]
            le = np.array(e, F)
            mat = (kd, ks, kt, F(t["Ni"]), le)
            if (le > 0).any():
                lights.append((p[0], p[1], p[2], mat))
                continue
            for k, other in enumerate(materials):
                if (all((np.abs(mat[i] - other[i]) <= EPS).all() for i in (0, 1, 2, 4))
                        and abs(mat[3] - other[3]) < EPS):
                    mat_index = k
                    break
            else:
                mat_index = len(materials)
                materials.append(mat)
        if not has_normal:   # Triangle.cpp:10-17
            g = _normalize(_cross(p[2] - p[0], p[1] - p[0]))
            n = [g, g, g]
        abc.append(np.concatenate(p))
        normals.append(np.concatenate(n))
        colors.append(np.concatenate(cc))
        tmat.append(mat_index)
    shape = (len(abc), 9)
    return (np.array(abc, F).reshape(shape), np.array(normals, F).reshape(shape), np.array(colors, F).reshape(shape),
            np.array(tmat, np.int32), materials, lights)
