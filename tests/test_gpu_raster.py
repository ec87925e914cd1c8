"""The raster preview on the device (mrt_raster_preview) against the oracle's restatement, bit for bit:
Cornell box (Perspective and Orthographic), terrain, a 200,000-triangle soup, a scene whose triangles
cross the near plane, an empty scene, a padded row pitch and the device-memory path (GPU)."""
import numpy as np
import pytest

import orc as O
from mobileraytracer_b200 import MrtError, Scene, capi, scenes

pytestmark = pytest.mark.gpu


def _check(ctx, sc, cam, w, h):
    g = Scene(ctx, sc)
    bm, st = g.raster_preview(cam, w, h)
    want, drawn, frags = O.raster_preview(sc, cam, w, h)
    assert st.triangles == sc.n_triangles
    assert (st.drawn, st.fragments) == (drawn, frags)
    bad = np.argwhere(bm != want)
    assert len(bad) == 0, (len(bad), bad[:5], bm[tuple(bad[0])] if len(bad) else None)
    g.close()
    return bm, st


def test_cornell_perspective_and_orthographic(ctx):
    sc = scenes.cornell_box()
    bm, st = _check(ctx, sc, sc.camera, 256, 256)
    assert st.drawn > 0 and (bm != 0).all()   # the walls fill the frame
    ortho = scenes.orthographic((0.0, 0.0, -1.7), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 1.6, 1.2)
    _check(ctx, sc, ortho, 200, 150)


def test_terrain_and_soup(ctx):
    t = scenes.heightfield(cells=128, seed=1, width=384, height=256)
    _check(ctx, t, t.camera, 384, 256)
    s = scenes.triangle_soup(200_000, 3, 640, 360)
    bm, st = _check(ctx, s, s.camera, 640, 360)
    assert st.drawn > 50_000 and st.fragments > 0


def test_near_plane_crossing_and_large_triangles(ctx):
    # a floor and walls running from behind the camera to far in front: every triangle is clipped
    # against the near plane, and most cover thousands of pixels (the block-per-triangle path)
    sc = scenes.Scene()
    quads = []
    for (a, b, c, d) in (((-5, -1, -10), (5, -1, -10), (5, -1, 40), (-5, -1, 40)),
                         ((-2, -5, -10), (-2, -5, 40), (-2, 5, 40), (-2, 5, -10)),
                         ((2, 5, -10), (2, 5, 40), (2, -5, 40), (2, -5, -10))):
        quads += [list(a) + list(b) + list(c), list(a) + list(c) + list(d)]
    sc.tri_abc = np.asarray(quads, np.float32)
    sc.tri_material = np.full(len(quads), -1, np.int32)
    sc.tri_colors = np.repeat(np.asarray([[0.9, 0.2, 0.1], [0.1, 0.8, 0.3], [0.2, 0.3, 0.9], [0.5, 0.5, 0.5],
                                          [0.7, 0.1, 0.7], [0.1, 0.6, 0.6]], np.float32), 3, axis=0).reshape(-1, 9)
    cam = scenes.camera((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 60.0, 45.0)
    bm, st = _check(ctx, sc, cam, 320, 240)
    assert st.drawn >= 12 and st.fragments > 50_000   # a corridor: floor and both walls
    cam2 = scenes.camera((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 60.0, 45.0)   # looking back
    _check(ctx, sc, cam2, 320, 240)


def test_empty_scene_padded_pitch_and_device_path(ctx):
    torch = pytest.importorskip("torch")
    empty = scenes.Scene()
    cam = scenes.camera((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    bm, st = _check(ctx, empty, cam, 64, 48)
    assert not bm.any() and st.drawn == 0
    sc = scenes.cornell_box()
    g = Scene(ctx, sc)
    want, _, _ = O.raster_preview(sc, sc.camera, 128, 96)
    # host bitmap with 16 pixels of row padding that the preview must leave alone
    padded = np.full((96, 144), 0xDEADBEEF, np.uint32)
    g.raster_preview(sc.camera, 128, 96, bitmap=padded, stride_bytes=144 * 4)
    assert (padded[:, :128] == want).all() and (padded[:, 128:] == 0xDEADBEEF).all()
    dev = torch.zeros((96, 128), dtype=torch.int32, device="cuda")
    g.raster_preview(sc.camera, 128, 96, bitmap=dev)
    torch.cuda.synchronize()
    assert (dev.cpu().numpy().view(np.uint32) == want).all()
    g.close()


def test_invalid_arguments(ctx):
    sc = scenes.cornell_box()
    g = Scene(ctx, sc)
    bad = scenes.camera((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), fov_h=0.0)
    with pytest.raises(MrtError):
        g.raster_preview(bad, 64, 64)
    with pytest.raises(MrtError):
        g.raster_preview(sc.camera, 9000, 64)
    g.close()


def test_pixel_centre_edges_and_guard_band(ctx):
    # shared edges exactly through pixel centres (the top-left rule decides) and a triangle reaching
    # far beyond the guard band: the device equals the restatement bit for bit
    cam = scenes.orthographic((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 16.0, 16.0)
    ring = [(-3.875, -3.875), (3.875, -3.875), (3.875, 3.875), (-3.875, 3.875)]
    sc = scenes.Scene()
    sc.tri_abc = np.asarray([[0.125, 0.125, 0.0, *ring[k], 0.0, *ring[(k + 1) % 4], 0.0] for k in range(4)], np.float32)
    sc.tri_material = np.full(4, -1, np.int32)
    sc.tri_colors = np.asarray([[1, 0, 0] * 3, [0, 1, 0] * 3, [1, 0, 0] * 3, [0, 1, 0] * 3], np.float32)
    bm, st = _check(ctx, sc, cam, 32, 32)
    assert st.fragments == 31 * 31
    big = scenes.Scene()
    big.tri_abc = np.asarray([[-500, -500, 0, 500, -500, 0, 0, 500, 0]], np.float32)
    big.tri_material = np.full(1, -1, np.int32)
    big.tri_colors = np.asarray([[1, 0, 0] * 3], np.float32)
    bm, st = _check(ctx, big, scenes.camera((0.0, 0.0, -3.0), (0.0, 0.0, 0.0)), 40, 30)
    assert st.fragments == 40 * 30


def test_vertices_at_near_plane_and_guard_band_corners(ctx):
    # one vertex of every triangle at a corner of the near plane and the guard band: the device clipper
    # equals the restatement bit for bit (bitmap, drawn triangles, covered samples)
    from helpers import near_guard_corner_scene
    sc, cam, w, h = near_guard_corner_scene()
    _check(ctx, sc, cam, w, h)


def test_full_queue_sends_triangles_to_further_passes(ctx, monkeypatch):
    """Large pieces beyond the queue's room: the triangles owning them are drawn whole by further
    passes over an overflow list.  With the room lowered to 14 entries (the pieces of one clipped
    triangle) the Cornell box, a 2,000-triangle soup and a clipped corridor still equal the oracle
    bit for bit, with the same drawn and covered counts."""
    monkeypatch.setenv("MRT_RASTER_QUEUE_CAP", "14")
    sc = scenes.cornell_box()
    _check(ctx, sc, sc.camera, 256, 256)
    s = scenes.triangle_soup(2_000, 4, 320, 240)
    _check(ctx, s, s.camera, 320, 240)
    quads = []
    for (a, b, c, d) in (((-5, -1, -10), (5, -1, -10), (5, -1, 40), (-5, -1, 40)),
                         ((-2, -5, -10), (-2, -5, 40), (-2, 5, 40), (-2, 5, -10))):
        quads += [list(a) + list(b) + list(c), list(a) + list(c) + list(d)]
    corridor = scenes.Scene()
    corridor.tri_abc = np.asarray(quads * 8, np.float32)   # 32 large clipped triangles in draw order
    corridor.tri_material = np.full(len(quads) * 8, -1, np.int32)
    corridor.tri_colors = np.tile(np.asarray([[0.9, 0.2, 0.1]], np.float32), (len(quads) * 8, 3))
    cam = scenes.camera((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 60.0, 45.0)
    _check(ctx, corridor, cam, 320, 240)
