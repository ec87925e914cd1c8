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
