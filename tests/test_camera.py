"""The host-side camera rays (mobileraytracer_b200.camera.primary_rays, used by the counting replay
behind the roofline figure) equal the oracle's Perspective::generateRay / Orthographic::generateRay
(Perspective.cpp:24-44, Orthographic.cpp:23-31) bit for bit."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from mobileraytracer_b200 import camera as mcam
from mobileraytracer_b200 import capi, scenes

from helpers import camera_rays


def _orc_rays(cam, width, height, pixels):
    import orc as O
    lib = O.orc()
    out = np.zeros(6, np.float32)
    res = np.zeros((len(pixels), 6), np.float32)
    inv_w, inv_h = np.float32(1.0) / np.float32(width), np.float32(1.0) / np.float32(height)
    for k, p in enumerate(pixels):
        u, v = np.float32(p % width) * inv_w, np.float32(p // width) * inv_h
        lib.orc_camera_ray(ctypes.byref(cam), float(u), float(v), 0.0, 0.0, O.fptr(out))
        res[k] = out
    return res


def test_perspective_rays_of_the_1080p_frame():
    sc = scenes.triangle_soup(64, 0, 1920, 1080)
    step = 997
    ours = mcam.primary_rays(sc.camera, 1920, 1080, pixels=np.arange(0, 1920 * 1080, step))
    ref = camera_rays(sc.camera, 1920, 1080, step=step)
    assert np.array_equal(ours["origin"].view(np.uint32), ref["origin"].view(np.uint32))
    assert np.array_equal(ours["direction"].view(np.uint32), ref["direction"].view(np.uint32))


@pytest.mark.parametrize("kind", ["perspective", "orthographic"])
def test_camera_kinds_on_the_cornell_box(kind):
    sc = scenes.cornell_box()
    cam = sc.camera
    if kind == "orthographic":
        cam = capi.MrtCamera(kind=capi.MRT_CAMERA_ORTHOGRAPHIC, position=cam.position, look_at=cam.look_at,
                             up=cam.up, fov_h_deg=1.2, fov_v_deg=1.2)
    pix = np.arange(0, 96 * 80, 37)
    ours = mcam.primary_rays(cam, 96, 80, pixels=pix)
    ref = _orc_rays(cam, 96, 80, pix)
    assert np.array_equal(ours["origin"].view(np.uint32), ref[:, :3].view(np.uint32))
    assert np.array_equal(ours["direction"].view(np.uint32), ref[:, 3:].view(np.uint32))
