"""Shared helpers for the parity tests: seeded rays and hit comparisons."""
from __future__ import annotations

import ctypes

import numpy as np

from mobileraytracer_b200 import capi, scenes

RAY_DTYPE = np.dtype([("origin", np.float32, 3), ("direction", np.float32, 3), ("depth", np.int32),
                      ("exclude", np.uint32)])


def random_rays(n: int, seed: int = 5, lo: float = -0.9, hi: float = 0.9, inside: bool = True) -> np.ndarray:
    """Rays with origins uniform in [lo, hi]^3 and uniform random unit directions."""
    u = scenes.uniform(seed, n * 6).reshape(n, 6)
    o = lo + (hi - lo) * u[:, :3]
    d = 2.0 * u[:, 3:] - 1.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros(n, RAY_DTYPE)
    r["origin"] = o.astype(np.float32)
    r["direction"] = d.astype(np.float32)
    r["depth"] = 1
    r["exclude"] = 0xFFFFFFFF
    return r


def camera_rays(cam: capi.MrtCamera, width: int, height: int, step: int = 1, first: int = 0) -> np.ndarray:
    """Camera rays of Renderer::renderScene for every `step`-th pixel, Constant(0.5) jitter, from
    the oracle's restatement of Perspective::generateRay."""
    import orc as O
    lib = O.orc()
    pix = np.arange(first, width * height, step)
    r = np.zeros(len(pix), RAY_DTYPE)
    out = np.zeros(6, np.float32)
    inv_w, inv_h = np.float32(1.0) / np.float32(width), np.float32(1.0) / np.float32(height)
    for k, p in enumerate(pix):
        x, y = int(p % width), int(p // width)
        u, v = np.float32(x) * inv_w, np.float32(y) * inv_h
        lib.orc_camera_ray(ctypes.byref(cam), float(u), float(v), 0.0, 0.0, O.fptr(out))
        r[k]["origin"] = out[:3]
        r[k]["direction"] = out[3:]
    r["depth"] = 1
    r["exclude"] = 0xFFFFFFFF
    return r


def hits_equal(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-ray equality of (id, t bits)."""
    return (a["id"] == b["id"]) & (a["t"].view(np.uint32) == b["t"].view(np.uint32))


def near_tie_mask(rays: np.ndarray, a: np.ndarray, b: np.ndarray, rel: float = 1e-6) -> np.ndarray:
    """Rays whose two answers are both hits with distances within `rel` of each other: a tie the
    spec counts separately (the id may legitimately differ)."""
    both = (a["id"] != capi.MRT_HIT_NONE) & (b["id"] != capi.MRT_HIT_NONE)
    ta, tb = a["t"].astype(np.float64), b["t"].astype(np.float64)
    return both & (np.abs(ta - tb) <= rel * np.maximum(np.abs(ta), np.abs(tb)))


def near_guard_corner_scene(seed: int = 11, per_corner: int = 40, w: int = 160, h: int = 120):
    """Triangles with one vertex within 1e-4 (relative) of a corner where the near plane (0.1) meets
    the raster preview's guard band (16 viewports) for a camera at the origin looking along +z with a
    45-degree vertical field of view, the other vertices in front of and behind the near plane: the
    clipper meets near-coincident planes, where rounded intersection points can add vertices."""
    from mobileraytracer_b200 import scenes
    rng = np.random.default_rng(seed)
    cam = scenes.camera((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 60.0, 45.0)
    t = np.tan(np.radians(0.918 * 45.0) / 2.0)
    tris = []
    for sx in (-1.0, 1.0):
        for sy in (-1.0, 1.0):
            corner = np.array([sx * 16.0 * 0.1 * t * w / h, sy * 16.0 * 0.1 * t, 0.1])
            for _ in range(per_corner):
                a = corner * (1.0 + rng.uniform(-1e-4, 1e-4, 3))
                b = rng.uniform([-2.0, -2.0, 0.5], [2.0, 2.0, 5.0])
                c = rng.uniform([-2.0, -2.0, -1.0], [2.0, 2.0, 0.05])
                tris.append([*a, *b, *c] if rng.random() < 0.5 else [*a, *c, *b])
    sc = scenes.Scene()
    sc.tri_abc = np.asarray(tris, np.float32)
    n = len(tris)
    sc.tri_material = np.full(n, -1, np.int32)
    sc.tri_colors = rng.uniform(0.1, 1.0, (n, 9)).astype(np.float32)
    return sc, cam, w, h
