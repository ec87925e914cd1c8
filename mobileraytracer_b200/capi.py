"""ctypes mirror of include/mrt_cuda.h and the loader of the CUDA library.

The structures here must match the C header field for field; tests/test_capi_layout.py checks the
sizes against the compiled library.  Loading fails loudly: there is no CPU fallback for any entry
point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MRT_CUDA_LIB") or os.path.join(HERE, "lib", "libmrt_cuda.so")

MRT_OK, MRT_ERR_ARG, MRT_ERR_OOM, MRT_ERR_CUDA, MRT_ERR_LIMIT, MRT_ERR_CANCELLED, MRT_ERR_STATE = range(7)
MRT_ACCEL_NAIVE, MRT_ACCEL_REGULAR_GRID, MRT_ACCEL_BVH = 0, 1, 2
MRT_BVH_FAST, MRT_BVH_REFERENCE = 0, 1
MRT_GRID_INDEX_REFERENCE, MRT_GRID_INDEX_LINEAR = 0, 1
MRT_SHADER_NOSHADOWS, MRT_SHADER_WHITTED, MRT_SHADER_PATHTRACER, MRT_SHADER_DEPTHMAP, MRT_SHADER_DIFFUSE = 0, 1, 2, 3, 4
MRT_SAMPLER_CONSTANT, MRT_SAMPLER_STRATIFIED, MRT_SAMPLER_HALTON, MRT_SAMPLER_RANDOM = 0, 1, 2, 3
MRT_LIGHT_POINT, MRT_LIGHT_AREA = 0, 1
MRT_CAMERA_PERSPECTIVE, MRT_CAMERA_ORTHOGRAPHIC = 0, 1
MRT_PRIM_PLANE, MRT_PRIM_SPHERE, MRT_PRIM_TRIANGLE, MRT_PRIM_LIGHT = 0, 1, 2, 3
MRT_HIT_NONE = 0xFFFFFFFF
MRT_MEM_HOST, MRT_MEM_DEVICE = 0, 1
MRT_BATCH_SMALLEST_FIRST, MRT_BATCH_FIFO, MRT_BATCH_EQUAL_SHARE = 0, 1, 2
MRT_BATCH_KERNEL_WAVEFRONT, MRT_BATCH_KERNEL_PATHS = 1, 2
MRT_RENDER_SHADE_QUEUES = 1
RAY_LENGTH_MAX = 1.0e30

STATUS_NAMES = {0: "MRT_OK", 1: "MRT_ERR_ARG", 2: "MRT_ERR_OOM", 3: "MRT_ERR_CUDA", 4: "MRT_ERR_LIMIT",
                5: "MRT_ERR_CANCELLED", 6: "MRT_ERR_STATE"}


def hit_id(prim_type: int, index: int) -> int:
    return ((prim_type & 3) << 30) | (index & 0x3FFFFFFF)


class MrtMaterial(ctypes.Structure):
    _fields_ = [("le", ctypes.c_float * 3), ("kd", ctypes.c_float * 3), ("ks", ctypes.c_float * 3),
                ("kt", ctypes.c_float * 3), ("ior", ctypes.c_float)]


class MrtLightDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("p0", ctypes.c_float * 3), ("p1", ctypes.c_float * 3),
                ("p2", ctypes.c_float * 3), ("radiance", MrtMaterial)]


class MrtSceneDesc(ctypes.Structure):
    _fields_ = [
        ("n_triangles", ctypes.c_uint32),
        ("tri_abc", ctypes.POINTER(ctypes.c_float)),
        ("tri_normals", ctypes.POINTER(ctypes.c_float)),
        ("tri_colors", ctypes.POINTER(ctypes.c_float)),
        ("tri_material", ctypes.POINTER(ctypes.c_int32)),
        ("n_spheres", ctypes.c_uint32),
        ("sphere_center_radius", ctypes.POINTER(ctypes.c_float)),
        ("sphere_material", ctypes.POINTER(ctypes.c_int32)),
        ("n_planes", ctypes.c_uint32),
        ("plane_point_normal", ctypes.POINTER(ctypes.c_float)),
        ("plane_material", ctypes.POINTER(ctypes.c_int32)),
        ("n_materials", ctypes.c_uint32),
        ("materials", ctypes.POINTER(MrtMaterial)),
        ("n_lights", ctypes.c_uint32),
        ("lights", ctypes.POINTER(MrtLightDesc)),
    ]


class MrtCamera(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("position", ctypes.c_float * 3), ("look_at", ctypes.c_float * 3),
                ("up", ctypes.c_float * 3), ("fov_h_deg", ctypes.c_float), ("fov_v_deg", ctypes.c_float)]


class MrtAccelOpts(ctypes.Structure):
    _fields_ = [("accelerator", ctypes.c_int32), ("bvh_mode", ctypes.c_int32), ("grid_size", ctypes.c_int32),
                ("grid_index", ctypes.c_int32), ("camera_position", ctypes.c_float * 3),
                ("camera", ctypes.POINTER(MrtCamera))]


class MrtRay(ctypes.Structure):
    _fields_ = [("origin", ctypes.c_float * 3), ("direction", ctypes.c_float * 3), ("depth", ctypes.c_int32),
                ("exclude", ctypes.c_uint32)]


class MrtHit(ctypes.Structure):
    _fields_ = [("t", ctypes.c_float), ("id", ctypes.c_uint32)]


class MrtRenderOpts(ctypes.Structure):
    _fields_ = [
        ("shader", ctypes.c_int32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
        ("spp", ctypes.c_uint32), ("spl", ctypes.c_uint32), ("pixel_sampler", ctypes.c_int32),
        ("constant_value", ctypes.c_float), ("light_sampler", ctypes.c_int32), ("rr_sampler", ctypes.c_int32),
        ("depth_min", ctypes.c_int32), ("depth_max", ctypes.c_int32), ("seed", ctypes.c_uint64),
        ("spp_offset", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("depth_point", ctypes.c_float * 3),
        ("reserved2", ctypes.c_uint32),
    ]


class MrtRenderStats(ctypes.Structure):
    _fields_ = [("rays_closest", ctypes.c_uint64), ("rays_shadow", ctypes.c_uint64), ("paths", ctypes.c_uint64),
                ("device_ms", ctypes.c_float), ("trace_ms", ctypes.c_float), ("kernel_launches", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class MrtRasterStats(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_uint64), ("drawn", ctypes.c_uint64), ("fragments", ctypes.c_uint64),
                ("device_ms", ctypes.c_float)]


class MrtBatchOpts(ctypes.Structure):
    _fields_ = [("wave_roots", ctypes.c_uint32), ("block_threads", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32), ("max_jobs", ctypes.c_uint32), ("max_depth", ctypes.c_uint32),
                ("max_spl", ctypes.c_uint32), ("no_graph", ctypes.c_uint32), ("max_wave_roots", ctypes.c_uint32),
                ("policy", ctypes.c_uint32), ("pipelines", ctypes.c_uint32), ("kernel", ctypes.c_uint32)]


class MrtBatchJob(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("camera", MrtCamera), ("opts", MrtRenderOpts),
                ("bitmap", ctypes.c_void_p), ("stride_bytes", ctypes.c_uint32), ("accum", ctypes.c_void_p)]


class MrtBatchStats(ctypes.Structure):
    _fields_ = [("rays_closest", ctypes.c_uint64), ("rays_shadow", ctypes.c_uint64), ("paths", ctypes.c_uint64),
                ("waves", ctypes.c_uint64), ("jobs_submitted", ctypes.c_uint64), ("jobs_done", ctypes.c_uint64),
                ("busy_ms", ctypes.c_double), ("wave_roots", ctypes.c_uint32), ("block_threads", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32), ("autotuned", ctypes.c_uint32), ("pipelines", ctypes.c_uint32),
                ("kernel", ctypes.c_uint32), ("waves_paths", ctypes.c_uint64)]


class MrtServeOpts(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_uint64), ("build_slack_bytes", ctypes.c_uint64), ("batch", MrtBatchOpts)]


class MrtServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("builds", ctypes.c_uint64),
                ("evictions", ctypes.c_uint64), ("resident_bytes", ctypes.c_uint64), ("peak_bytes", ctypes.c_uint64),
                ("rays_closest", ctypes.c_uint64), ("rays_shadow", ctypes.c_uint64)]


def render_opts(shader=MRT_SHADER_NOSHADOWS, width=256, height=256, spp=1, spl=1, pixel_sampler=None,
                constant_value=0.5, light_sampler=MRT_SAMPLER_RANDOM, rr_sampler=MRT_SAMPLER_RANDOM,
                depth_min=4, depth_max=8, seed=0, spp_offset=0, depth_point=(1.0, 1.0, 1.0), flags=0) -> MrtRenderOpts:
    """Options with the reference CLI's wiring as defaults (c_wrapper.cpp:436-443,455): the pixel
    sampler is Constant(0.5) at 1 spp and random otherwise; RayDepthMin 4, RayDepthMax 8."""
    if pixel_sampler is None:
        pixel_sampler = MRT_SAMPLER_CONSTANT if spp <= 1 else MRT_SAMPLER_RANDOM
    o = MrtRenderOpts()
    o.shader, o.width, o.height, o.spp, o.spl = shader, width, height, spp, spl
    o.pixel_sampler, o.constant_value = pixel_sampler, constant_value
    o.light_sampler, o.rr_sampler = light_sampler, rr_sampler
    o.depth_min, o.depth_max, o.seed, o.spp_offset = depth_min, depth_max, seed, spp_offset
    o.depth_point[:] = depth_point
    o.flags = flags
    return o


_lib = None


def load() -> ctypes.CDLL:
    """Load libmrt_cuda.so and declare its signatures; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mobileraytracer_b200.build` "
                           "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    sig = {
        "mrt_context_create": (ctypes.c_int, [ctypes.c_int, P(vp)]),
        "mrt_context_destroy": (None, [vp]),
        "mrt_context_error": (ctypes.c_char_p, [vp]),
        "mrt_context_synchronize": (ctypes.c_int, [vp]),
        "mrt_context_stream": (vp, [vp]),
        "mrt_scene_create": (ctypes.c_int, [vp, P(MrtSceneDesc), P(vp)]),
        "mrt_scene_destroy": (None, [vp]),
        "mrt_scene_build": (ctypes.c_int, [vp, P(MrtAccelOpts)]),
        "mrt_scene_move": (ctypes.c_int, [vp, vp]),
        "mrt_scene_device_bytes": (ctypes.c_uint64, [vp]),
        "mrt_scene_accel_info": (ctypes.c_int, [vp, P(ctypes.c_uint64), P(ctypes.c_uint64), P(ctypes.c_int32)]),
        "mrt_trace_closest": (ctypes.c_int, [vp, vp, ctypes.c_uint32, vp, ctypes.c_uint32]),
        "mrt_trace_any": (ctypes.c_int, [vp, vp, vp, ctypes.c_uint32, vp, ctypes.c_uint32]),
        "mrt_trace_closest_counts": (ctypes.c_int, [vp, vp, ctypes.c_uint32, vp, vp, ctypes.c_uint32]),
        "mrt_render": (ctypes.c_int, [vp, P(MrtCamera), P(MrtRenderOpts), vp, ctypes.c_uint32, vp, ctypes.c_uint32,
                                      P(MrtRenderStats)]),
        "mrt_render_noalloc": (ctypes.c_int, [vp, P(MrtCamera), P(MrtRenderOpts), vp, ctypes.c_uint32, vp,
                                              P(MrtRenderStats)]),
        "mrt_batch_create": (ctypes.c_int, [vp, P(MrtBatchOpts), P(vp)]),
        "mrt_batch_destroy": (None, [vp]),
        "mrt_batch_submit": (ctypes.c_int, [vp, P(MrtBatchJob), P(ctypes.c_uint64)]),
        "mrt_batch_step": (ctypes.c_int, [vp, ctypes.c_uint32, P(ctypes.c_uint32)]),
        "mrt_batch_completed": (ctypes.c_int, [vp, P(ctypes.c_uint64), ctypes.c_uint32, P(ctypes.c_uint32)]),
        "mrt_batch_run": (ctypes.c_int, [vp]),
        "mrt_batch_stats": (ctypes.c_int, [vp, P(MrtBatchStats)]),
        "mrt_arena_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, P(vp)]),
        "mrt_arena_destroy": (ctypes.c_int, [vp]),
        "mrt_arena_stats": (ctypes.c_int, [vp, P(ctypes.c_uint64), P(ctypes.c_uint64), P(ctypes.c_uint64),
                                           P(ctypes.c_uint64)]),
        "mrt_context_set_arena": (ctypes.c_int, [vp, vp]),
        "mrt_obj_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, P(vp), P(MrtSceneDesc), ctypes.c_char_p,
                                        ctypes.c_size_t]),
        "mrt_obj_free": (None, [vp]),
        "mrt_render_stop": (None, [vp]),
        "mrt_render_progress": (ctypes.c_uint32, [vp]),
        "mrt_raster_preview": (ctypes.c_int, [vp, P(MrtCamera), ctypes.c_uint32, ctypes.c_uint32, vp, ctypes.c_uint32,
                                              ctypes.c_uint32, P(MrtRasterStats)]),
        "mrt_serve_create": (ctypes.c_int, [ctypes.c_int, P(MrtServeOpts), P(vp)]),
        "mrt_serve_destroy": (None, [vp]),
        "mrt_serve_error": (ctypes.c_char_p, [vp]),
        "mrt_serve_add_scene": (ctypes.c_int, [vp, P(MrtSceneDesc), P(MrtAccelOpts), P(ctypes.c_uint64)]),
        "mrt_serve_submit": (ctypes.c_int, [vp, ctypes.c_uint64, P(MrtCamera), P(MrtRenderOpts), vp,
                                            P(ctypes.c_uint64)]),
        "mrt_serve_poll": (ctypes.c_int, [vp, P(ctypes.c_uint64), ctypes.c_uint32, P(ctypes.c_uint32)]),
        "mrt_serve_pending": (ctypes.c_int, [vp, P(ctypes.c_uint64)]),
        "mrt_serve_request_latency": (ctypes.c_int, [vp, ctypes.c_uint64, P(ctypes.c_double)]),
        "mrt_serve_stats": (ctypes.c_int, [vp, P(MrtServeStats)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


EXPORTED_SYMBOLS = [
    "mrt_context_create", "mrt_context_destroy", "mrt_context_error", "mrt_context_synchronize",
    "mrt_context_stream", "mrt_scene_create", "mrt_scene_destroy", "mrt_scene_build", "mrt_scene_device_bytes",
    "mrt_scene_accel_info", "mrt_trace_closest", "mrt_trace_any", "mrt_trace_closest_counts", "mrt_render",
    "mrt_render_noalloc", "mrt_render_stop", "mrt_render_progress", "mrt_batch_create", "mrt_batch_destroy",
    "mrt_batch_submit", "mrt_batch_step", "mrt_batch_completed", "mrt_batch_run", "mrt_batch_stats",
    "mrt_arena_create", "mrt_arena_destroy", "mrt_arena_stats", "mrt_context_set_arena", "mrt_scene_move",
    "mrt_obj_load", "mrt_obj_free", "mrt_raster_preview", "mrt_serve_create", "mrt_serve_destroy", "mrt_serve_error",
    "mrt_serve_add_scene", "mrt_serve_submit", "mrt_serve_poll", "mrt_serve_pending", "mrt_serve_request_latency",
    "mrt_serve_stats",
]
