"""Camera rays of Renderer::renderScene on the host, vectorised in float32.

Used to feed mrt_trace_closest / mrt_trace_closest_counts with exactly the rays the render kernels
generate (e.g. for the counting replay behind the roofline figure).  numpy float32 operations are
IEEE binary32 with no fused multiply-add, so with the reference's operation order the rays equal the
device ones bit for bit (tests/test_camera.py compares them with the oracle's camera):
  Camera ctor (Camera.cpp:52-57), Perspective ctor and generateRay / fastArcTan
  (Perspective.cpp:10-44), Orthographic ctor and generateRay (Orthographic.cpp:12-34), pixel loop
  u = x / W, v = y / H (Renderer.cpp:94-104).
"""
from __future__ import annotations

import numpy as np

from . import capi

F = np.float32


def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - b[..., 1] * a[..., 2],
                     a[..., 2] * b[..., 0] - b[..., 2] * a[..., 0],
                     a[..., 0] * b[..., 1] - b[..., 0] * a[..., 1]], -1)


def _normalize(v):
    inv = F(1.0) / np.sqrt(_dot(v, v))
    return v * inv[..., None]


def _fast_arctan(x):
    ax = np.abs(x)
    return F(0.785398163397448309616) * x - (x * (ax - F(1.0))) * (F(0.2447) + (F(0.0663) * ax))


def basis(cam: capi.MrtCamera):
    pos = np.asarray(cam.position, F)
    direction = _normalize(np.asarray(cam.look_at, F) - pos)
    right = _cross(np.asarray(cam.up, F), direction)
    up = _cross(direction, right)
    pi = F(3.14159265358979323846)
    hfov = (F(cam.fov_h_deg) * pi) / F(180.0)
    vfov = (F(cam.fov_v_deg) * pi) / F(180.0)
    return pos, direction, right, up, hfov, vfov


def primary_rays(cam: capi.MrtCamera, width: int, height: int, pixels: np.ndarray | None = None,
                 jitter: float = 0.5) -> np.ndarray:
    """MrtRay records for the given pixel indices (row-major, default all) with a Constant(jitter)
    camera sampler (the reference CLI's choice at 1 spp)."""
    from . import RAY_DTYPE
    if pixels is None:
        pixels = np.arange(width * height, dtype=np.int64)
    x = (pixels % width).astype(F)
    y = (pixels // width).astype(F)
    inv_w, inv_h = F(1.0) / F(width), F(1.0) / F(height)
    pw, ph = F(0.5) / F(width), F(0.5) / F(height)
    u, v = x * inv_w, y * inv_h
    j = F(jitter)
    du = (j - F(0.5)) * F(2.0) * pw
    dv = (j - F(0.5)) * F(2.0) * ph
    pos, direction, right, up, hfov, vfov = basis(cam)
    r = np.zeros(len(pixels), RAY_DTYPE)
    r["depth"] = 1
    r["exclude"] = 0xFFFFFFFF
    if cam.kind == capi.MRT_CAMERA_ORTHOGRAPHIC:   # Orthographic.cpp:12-34
        sh, sv = F(cam.fov_h_deg) / F(2.0), F(cam.fov_v_deg) / F(2.0)
        rgt = right[None, :] * ((u - F(0.5)) * sh)[:, None] + right[None, :] * du
        upv = up[None, :] * ((F(0.5) - v) * sv)[:, None] + up[None, :] * dv
        r["origin"] = ((pos[None, :] + rgt) + upv).astype(F)
        r["direction"] = direction
        return r
    rf = _fast_arctan(hfov * (u - F(0.5))) + du
    uf = _fast_arctan(vfov * (F(0.5) - v)) + dv
    dest = ((pos + direction)[None, :] + right[None, :] * rf[:, None]) + up[None, :] * uf[:, None]
    d = _normalize(dest - pos[None, :])
    r["origin"] = pos
    r["direction"] = d.astype(F)
    return r
