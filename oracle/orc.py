"""ctypes bindings of the oracle libraries.  TEST INFRASTRUCTURE ONLY (tests/, smoke(), bench.py's
cpu_baseline leg): the checker, never the product.

  liborc.so            the C restatement (oracle/orc.c)
  liboracle_ref.so     the reference's own sources compiled by oracle/Makefile (parity flags)
  liboracle_ref_fast.so  the same sources with the reference's release optimisation (CPU timing)
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_orc = None
_ref = {}


def _declare(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def orc() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        path = os.path.join(REF_DIR, "liborc.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle orc`")
        lib = ctypes.CDLL(path)
        vp, fp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int
        _declare(lib, {
            "orc_scene_create": (vp, [vp]),
            "orc_scene_destroy": (None, [vp]),
            "orc_scene_build": (ip, [vp, ip, ip, ip, fp]),
            "orc_scene_build_box": (ip, [vp, ip, ip, ip, fp, fp]),
            "orc_camera_box": (None, [vp, fp, fp]),
            "orc_scene_grid_size": (ip, [vp, ip]),
            "orc_scene_bvh_nodes": (ctypes.c_uint64, [vp, ip]),
            "orc_trace_closest": (None, [vp, vp, ctypes.c_uint32, vp, ip]),
            "orc_trace_any": (None, [vp, vp, vp, ctypes.c_uint32, vp, ip]),
            "orc_grid_counts": (ip, [vp, vp, ctypes.c_uint32, vp, vp, ip]),
            "orc_render": (ip, [vp, vp, vp, vp, ctypes.c_uint32, vp, vp, ip]),
            "orc_render_pixels": (ip, [vp, vp, vp, vp, ctypes.c_uint32, vp, ip]),
            "orc_triangle_intersect": (ip, [fp, fp, fp, fp, fp, ctypes.c_float, fp, fp, fp]),
            "orc_triangle_occludes": (ip, [fp, fp, fp, ctypes.c_float]),
            "orc_triangle_intersect_box": (ip, [fp, fp, fp]),
            "orc_plane_intersect_box": (ip, [fp, fp, fp]),
            "orc_plane_distance": (ctypes.c_float, [fp, fp]),
            "orc_plane_intersect": (ip, [fp, fp, fp, ctypes.c_float, fp]),
            "orc_sphere_intersect": (ip, [fp, fp, fp, ctypes.c_float, fp, fp]),
            "orc_sphere_intersect_box": (ip, [fp, fp, fp]),
            "orc_aabb_intersect": (ip, [fp, fp, fp, fp]),
            "orc_aabb_area": (ctypes.c_float, [fp, fp]),
            "orc_halton": (ctypes.c_float, [ctypes.c_uint32, ctypes.c_uint32]),
            "orc_incremental_avg": (ctypes.c_uint32, [fp, ctypes.c_uint32, ctypes.c_uint32]),
            "orc_camera_ray": (None, [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, fp]),
            "orc_sample": (ctypes.c_float, [vp, ip, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
            "orc_sincos": (None, [ctypes.c_float, fp, fp]),
            "orc_raster_preview": (ip, [vp, vp, ctypes.c_uint32, ctypes.c_uint32, vp, ctypes.c_uint32, vp]),
        })
        _orc = lib
    return _orc


def ref(fast: bool = False) -> ctypes.CDLL:
    key = "fast" if fast else "parity"
    if key not in _ref:
        path = os.path.join(REF_DIR, "liboracle_ref_fast.so" if fast else "liboracle_ref.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle ref` where the reference checkout exists")
        lib = ctypes.CDLL(path)
        vp, fp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int
        dp = ctypes.POINTER(ctypes.c_double)
        _declare(lib, {
            "ref_abi_version": (ip, []),
            "ref_triangle_intersect": (ip, [fp, fp, fp, fp, fp, ctypes.c_float, fp, fp, fp]),
            "ref_triangle_occludes": (ip, [fp, fp, fp, ctypes.c_float]),
            "ref_triangle_intersect_box": (ip, [fp, fp, fp]),
            "ref_triangle_fields": (None, [fp, fp]),
            "ref_plane_intersect_box": (ip, [fp, fp, fp]),
            "ref_plane_distance": (ctypes.c_float, [fp, fp]),
            "ref_plane_intersect": (ip, [fp, fp, fp, ctypes.c_float, fp]),
            "ref_plane_aabb": (None, [fp, fp]),
            "ref_sphere_intersect": (ip, [fp, fp, fp, ctypes.c_float, fp, fp]),
            "ref_sphere_intersect_box": (ip, [fp, fp, fp]),
            "ref_aabb_intersect": (ip, [fp, fp, fp, fp]),
            "ref_aabb_area": (ctypes.c_float, [fp, fp]),
            "ref_halton": (ctypes.c_float, [ctypes.c_uint32, ctypes.c_uint32]),
            "ref_incremental_avg": (ctypes.c_uint32, [fp, ctypes.c_uint32, ctypes.c_uint32]),
            "ref_camera_ray": (None, [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, fp]),
            "ref_trace_create": (vp, [vp, ip, fp]),
            "ref_trace_destroy": (None, [vp]),
            "ref_trace_closest": (ip, [vp, vp, ctypes.c_uint32, vp, ip]),
            "ref_trace_any": (ip, [vp, vp, vp, ctypes.c_uint32, vp, ip]),
            "ref_render": (ip, [vp, vp, vp, ip, ip, vp, ctypes.c_uint32, dp, dp]),
            "ref_render_subset": (ctypes.c_uint64, [vp, vp, vp, ip, ip, ctypes.c_uint32, ctypes.c_uint32, vp, dp, dp]),
            "ref_obj_fill": (ip, [ctypes.c_char_p, ctypes.c_char_p, vp, vp, ctypes.c_uint32, vp, ctypes.c_uint32, vp,
                                  vp, ctypes.c_uint32, vp, ctypes.c_uint32, vp, vp, vp, vp]),
        })
        _ref[key] = lib
    return _ref[key]


def fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def f32(*vals) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(vals, np.float32).reshape(-1))


RAY_DTYPE = np.dtype([("origin", np.float32, 3), ("direction", np.float32, 3), ("depth", np.int32), ("exclude", np.uint32)])
HIT_DTYPE = np.dtype([("t", np.float32), ("id", np.uint32)])


def make_rays(origins: np.ndarray, dirs: np.ndarray, depth: int = 1, exclude=None) -> np.ndarray:
    r = np.zeros(len(origins), RAY_DTYPE)
    r["origin"] = origins
    r["direction"] = dirs
    r["depth"] = depth
    r["exclude"] = 0xFFFFFFFF if exclude is None else exclude
    return r


def raster_preview(scene, camera, width: int, height: int):
    """The restatement of the raster preview: (bitmap uint32 [height, width], drawn, fragments)."""
    desc = scene.desc()
    bm = np.zeros((height, width), np.uint32)
    counts = np.zeros(2, np.uint64)
    st = orc().orc_raster_preview(ctypes.byref(desc), ctypes.byref(camera), width, height, bm.ctypes.data, width * 4,
                                  counts.ctypes.data)
    assert st == 0, st
    return bm, int(counts[0]), int(counts[1])


class OrcScene:
    """The restatement's scene with one accelerator built."""

    def __init__(self, scene, accel: int, grid_size: int = 0, grid_index: int = 0, camera_position=None,
                 camera=None):
        """Grid bounds include `camera`'s getAABB, else the point `camera_position`, else the
        scene's own camera (as Scene.build on the device side)."""
        self.lib = orc()
        self._scene = scene
        self._desc = scene.desc()
        self.h = self.lib.orc_scene_create(ctypes.byref(self._desc))
        if camera is None and camera_position is None and scene.camera is not None:
            camera = scene.camera
        if camera is not None:
            self._cmin, self._cmax = f32(0, 0, 0), f32(0, 0, 0)
            self.lib.orc_camera_box(ctypes.byref(camera), fptr(self._cmin), fptr(self._cmax))
            self.lib.orc_scene_build_box(self.h, accel, grid_size, grid_index, fptr(self._cmin), fptr(self._cmax))
        else:
            self._cam = f32(*(camera_position if camera_position is not None else [0.0, 0.0, 0.0]))
            self.lib.orc_scene_build(self.h, accel, grid_size, grid_index, fptr(self._cam))

    def close(self):
        if self.h:
            self.lib.orc_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def trace_closest(self, rays: np.ndarray, threads: int = 8) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        hits = np.zeros(len(rays), HIT_DTYPE)
        self.lib.orc_trace_closest(self.h, rays.ctypes.data, len(rays), hits.ctypes.data, threads)
        return hits

    def trace_any(self, rays: np.ndarray, dist: np.ndarray, threads: int = 8) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        dist = np.ascontiguousarray(dist, np.float32)
        occ = np.zeros(len(rays), np.uint8)
        self.lib.orc_trace_any(self.h, rays.ctypes.data, dist.ctypes.data, len(rays), occ.ctypes.data, threads)
        return occ

    def grid_counts(self, rays: np.ndarray, threads: int = 8):
        """(cells visited, triangle references tested) per ray by the triangle grid."""
        rays = np.ascontiguousarray(rays)
        cells = np.zeros(len(rays), np.uint32)
        refs = np.zeros(len(rays), np.uint32)
        assert self.lib.orc_grid_counts(self.h, rays.ctypes.data, len(rays), cells.ctypes.data, refs.ctypes.data,
                                        threads) == 0
        return cells, refs

    def render(self, camera, opts, threads: int = 8, bitmap=None, accum=None):
        w, h = opts.width, opts.height
        bm = np.zeros((h, w), np.uint32) if bitmap is None else bitmap
        acc = np.zeros((h, w, 4), np.float32) if accum is None else accum
        counts = np.zeros(2, np.uint64)
        st = self.lib.orc_render(self.h, ctypes.byref(camera), ctypes.byref(opts), bm.ctypes.data, w * 4,
                                 acc.ctypes.data, counts.ctypes.data, threads)
        assert st == 0, st
        return bm, acc, counts

    def render_pixels(self, camera, opts, xy: np.ndarray, threads: int = 8) -> np.ndarray:
        xy = np.ascontiguousarray(xy, np.uint32)
        out = np.zeros((len(xy), opts.spp, 3), np.float32)
        self.lib.orc_render_pixels(self.h, ctypes.byref(camera), ctypes.byref(opts), xy.ctypes.data, len(xy),
                                   out.ctypes.data, threads)
        return out


class RefScene:
    """The reference's own Shader::initializeAccelerators + rayTrace/shadowTrace."""

    def __init__(self, scene, accel: int, camera_position=None, fast: bool = False):
        self.lib = ref(fast)
        self._scene = scene
        self._desc = scene.desc()
        cam = camera_position if camera_position is not None else list(scene.camera.position)
        self._cam = f32(*cam)
        self.h = self.lib.ref_trace_create(ctypes.byref(self._desc), accel, fptr(self._cam))

    def close(self):
        if self.h:
            self.lib.ref_trace_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def trace_closest(self, rays: np.ndarray, threads: int = 8) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        hits = np.zeros(len(rays), HIT_DTYPE)
        self.lib.ref_trace_closest(self.h, rays.ctypes.data, len(rays), hits.ctypes.data, threads)
        return hits

    def trace_any(self, rays: np.ndarray, dist: np.ndarray, threads: int = 8) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        dist = np.ascontiguousarray(dist, np.float32)
        occ = np.zeros(len(rays), np.uint8)
        self.lib.ref_trace_any(self.h, rays.ctypes.data, dist.ctypes.data, len(rays), occ.ctypes.data, threads)
        return occ


def ref_render(scene, camera, opts, accel: int, threads: int = 8, fast: bool = False):
    lib = ref(fast)
    desc = scene.desc()
    bm = np.zeros((opts.height, opts.width), np.uint32)
    tb, tr = ctypes.c_double(), ctypes.c_double()
    lib.ref_render(ctypes.byref(desc), ctypes.byref(camera), ctypes.byref(opts), accel, threads, bm.ctypes.data,
                   opts.width * 4, ctypes.byref(tb), ctypes.byref(tr))
    return bm, tb.value, tr.value


def ref_render_subset(scene, camera, opts, accel: int, threads: int, first: int, step: int, fast: bool = True):
    lib = ref(fast)
    desc = scene.desc()
    total = opts.width * opts.height
    count = (total - first + step - 1) // step
    bm = np.zeros(count, np.uint32)
    tb, tr = ctypes.c_double(), ctypes.c_double()
    n = lib.ref_render_subset(ctypes.byref(desc), ctypes.byref(camera), ctypes.byref(opts), accel, threads, first,
                              step, bm.ctypes.data, ctypes.byref(tb), ctypes.byref(tr))
    return bm, int(n), tb.value, tr.value


def ref_obj_fill(obj_path: str, mtl_path: str | None, parsed):
    """OBJLoader::process + fillScene compiled from the reference sources, run on a staged parse
    (obj_oracle.parse's result).  Returns (triangles (n, 30) float32 with A, AB, AC, normals,
    colours and the material index as int bits in column 27, materials (m, 13) Le Kd Ks Kt ior,
    area lights (k, 22) A AB AC + material)."""
    pos, col, nrm, tris, mats = parsed
    lib = ref()
    v = np.ascontiguousarray(np.asarray(pos, np.float32).reshape(-1, 3))
    c = np.ascontiguousarray(np.asarray(col, np.float32).reshape(-1, 3))
    n = np.ascontiguousarray(np.asarray(nrm, np.float32).reshape(-1, 3)) if nrm else np.zeros((0, 3), np.float32)
    idx = np.ascontiguousarray(np.array([[a[0], a[1], b[0], b[1], cc[0], cc[1]] for a, b, cc, _ in tris],
                                        np.int32).reshape(-1, 6))
    fmat = np.ascontiguousarray(np.array([m for *_, m in tris], np.int32))
    mt = np.zeros((max(1, len(mats)), 14), np.float32)
    for k, m in enumerate(mats):
        mt[k, 0:3], mt[k, 3:6], mt[k, 6:9], mt[k, 9:12] = m["Kd"], m["Ks"], m["Kt"], m["Ke"]
        mt[k, 12], mt[k, 13] = m["Ni"], m["d"]
    nf = len(tris)
    out_tri = np.zeros((max(1, nf), 30), np.float32)
    out_mat = np.zeros((max(1, len(mats)), 13), np.float32)
    out_light = np.zeros((max(1, nf), 22), np.float32)
    counts = np.zeros(3, np.uint32)
    st = lib.ref_obj_fill(obj_path.encode(), mtl_path.encode() if mtl_path else None, v.ctypes.data, c.ctypes.data,
                          len(v), n.ctypes.data, len(n), idx.ctypes.data, fmat.ctypes.data, nf, mt.ctypes.data,
                          len(mats), out_tri.ctypes.data, out_mat.ctypes.data, out_light.ctypes.data, counts.ctypes.data)
    if st != 0:
        raise RuntimeError(f"ref_obj_fill failed: {st}")
    return out_tri[:counts[0]], out_mat[:counts[1]], out_light[:counts[2]]
