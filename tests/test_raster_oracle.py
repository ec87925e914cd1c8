"""The oracle's restatement of the raster preview (MainRenderer.copyFrame) on hand-made scenes: face
culling, depth order, tie rule, shared edges, near-plane clipping, colours (CPU only)."""
import numpy as np
import pytest

from mobileraytracer_b200 import scenes

orc = pytest.importorskip("oracle.orc")

CAM = scenes.camera((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0, 45.0)
RED, GREEN = [1.0, 0.0, 0.0] * 3, [0.0, 1.0, 0.0] * 3
PX_RED, PX_GREEN = 0xFF0000FF, 0xFF00FF00


def scene(tris, colors=None, mats=None, materials=()):
    s = scenes.Scene()
    s.tri_abc = np.asarray(tris, np.float32).reshape(-1, 9)
    n = len(s.tri_abc)
    s.tri_material = np.asarray(mats if mats is not None else [-1] * n, np.int32)
    if colors is not None:
        s.tri_colors = np.asarray(colors, np.float32).reshape(-1, 9)
    s.materials = list(materials)
    return s


def preview(s, w=32, h=32, cam=CAM):
    try:
        return orc.raster_preview(s, cam, w, h)
    except RuntimeError as e:   # liborc.so not built here
        pytest.skip(str(e))


def test_front_faces_drawn_back_faces_culled():
    front = [-1, -1, 0, 1, -1, 0, 0, 1, 0]
    back = [-1, -1, 0, 0, 1, 0, 1, -1, 0]
    bm, drawn, frags = preview(scene(front, RED))
    assert drawn == 1 and frags > 100 and frags == int((bm != 0).sum())
    assert bm[16, 16] == PX_RED
    # the apex (y = +1) is at the top of the bitmap: rows are flipped on read-back
    assert (bm[28] != 0).sum() > (bm[4] != 0).sum()
    bm, drawn, frags = preview(scene(back, RED))
    assert drawn == 0 and frags == 0 and not bm.any()


def test_nearest_wins_in_either_draw_order():
    near = [-1, -1, -0.5, 1, -1, -0.5, 0, 1, -0.5]
    far = [-1, -1, 0.5, 1, -1, 0.5, 0, 1, 0.5]
    for tris, cols, want in (((near, far), (RED, GREEN), PX_RED), ((far, near), (GREEN, RED), PX_RED)):
        bm, drawn, _ = preview(scene(tris, cols))
        assert drawn == 2 and bm[16, 16] == want


def test_depth_tie_goes_to_the_later_triangle():
    t = [-1, -1, 0, 1, -1, 0, 0, 1, 0]
    bm, _, frags = preview(scene([t, t], [RED, GREEN]))
    covered = bm != 0
    assert frags == 2 * int(covered.sum())
    assert (bm[covered] == PX_GREEN).all()


def test_shared_edge_covers_each_pixel_once():
    a, b, c, d = (-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)
    quad = [list(a) + list(b) + list(c), list(a) + list(c) + list(d)]
    bm, drawn, frags = preview(scene(quad, [RED, GREEN]), 48, 48)
    assert drawn == 2
    covered = int((bm != 0).sum())
    assert frags == covered   # no pixel centre counted by both triangles
    rows = np.nonzero((bm != 0).any(1))[0]
    cols = np.nonzero((bm != 0).any(0))[0]
    box = bm[rows[0]:rows[-1] + 1, cols[0]:cols[-1] + 1]
    assert (box != 0).all()   # and none missed inside the square


def test_triangle_through_the_near_plane_is_clipped():
    # from behind the camera (z = -4) to in front of it (z = +1): only the part in front is drawn
    t = [-1, -1, -4, 1, -1, -4, 0, -0.5, 1]
    bm, drawn, frags = preview(scene(t, RED))
    assert drawn >= 1 and frags > 0 and frags == int((bm != 0).sum())


def test_colours_material_max_and_vertex_mean():
    mat = scenes._material(le=(0.0, 0.0, 2.0), kd=(0.2, 0.5, 0.1), ks=(0.3, 0.1, 0.0))
    t = [-1, -1, 0, 1, -1, 0, 0, 1, 0]
    bm, _, _ = preview(scene(t, mats=[0], materials=[mat]))
    assert bm[16, 16] == (77 | 128 << 8 | 255 << 16 | 255 << 24)
    bm, _, _ = preview(scene(t, colors=[0.3, 0, 0, 0.6, 0, 0, 0, 0, 0.9]))
    f = np.float32
    r = ((f(0.3) + f(0.6)) + f(0.0)) / f(3.0)   # (cA + cB + cC) / 3 in float: 0.3 + 6e-8
    b = ((f(0.0) + f(0.0)) + f(0.9)) / f(3.0)   # 0.3 - 2e-8
    unorm = lambda c: int(f(c) * f(255.0) + f(0.5))
    assert (unorm(r), unorm(b)) == (77, 76)
    assert bm[16, 16] == (unorm(r) | 0 << 8 | unorm(b) << 16 | 255 << 24)


def test_orthographic_and_empty_scene():
    cam = scenes.orthographic((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 8.0, 8.0)
    # getSizeH returns the half size 4 and orthoM gets +-4 / 2: the view spans x, y in [-2, 2], so a
    # triangle 2 wide covers half of the 64 columns
    bm, drawn, frags = preview(scene([-1, -1, 0, 1, -1, 0, 0, 1, 0], RED), 64, 64, cam)
    cols = np.nonzero((bm != 0).any(0))[0]
    assert drawn == 1 and 31 <= len(cols) <= 33
    bm, drawn, frags = preview(scene(np.zeros((0, 9), np.float32)), 16, 16)
    assert drawn == 0 and frags == 0 and not bm.any()


def test_guard_band_and_degenerate_triangles():
    # a triangle reaching far outside the view in x and y (clipped by the guard band) still covers
    # every pixel of the frame it spans; a zero-area triangle draws nothing
    big = [-500, -500, 0, 500, -500, 0, 0, 500, 0]
    bm, drawn, frags = preview(scene(big, RED), 40, 30)
    assert drawn >= 1 and frags == 40 * 30 and (bm == PX_RED).all()
    flat = [-1, 0, 0, 1, 0, 0, 0.5, 0, 0]
    bm, drawn, frags = preview(scene(flat, RED))
    assert drawn == 0 and frags == 0 and not bm.any()


def test_edges_through_pixel_centres_are_owned_once():
    # an orthographic view whose pixel centres sit on the lines x = k / 4 (k odd) with the film
    # matched to the frame: a fan of triangles whose shared edges pass exactly through pixel centres
    cam = scenes.orthographic((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 16.0, 16.0)
    # view spans [-4, 4] over 32 pixels: centres at -4 + (i + 0.5) / 4
    c = (0.125, 0.125, 0.0)
    ring = [(-3.875, -3.875), (3.875, -3.875), (3.875, 3.875), (-3.875, 3.875)]
    tris = []
    for k in range(4):
        a, b = ring[k], ring[(k + 1) % 4]
        tris.append([c[0], c[1], 0.0, a[0], a[1], 0.0, b[0], b[1], 0.0])
    cols = [RED, GREEN, RED, GREEN]
    bm, drawn, frags = preview(scene(tris, cols), 32, 32, cam)
    assert drawn == 4
    assert frags == int((bm != 0).sum())   # every covered centre belongs to exactly one triangle
    assert frags == 31 * 31                # the square's centres, edges included once


def test_vertices_at_near_plane_and_guard_band_corners():
    # near-coincident clip planes: the clipper's polygon stays within its bound and the triangles
    # that reach the view are drawn
    from helpers import near_guard_corner_scene
    sc, cam, w, h = near_guard_corner_scene()
    bm, drawn, frags = preview(sc, w, h, cam)
    assert 0 < drawn <= sc.n_triangles and frags >= int((bm != 0).sum()) > 0   # frags: covered samples, overdraw included

