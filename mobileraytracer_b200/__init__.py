"""B200 render path for MobileRT (MobileRayTracer).

The work happens in CUDA kernels behind the C ABI of include/mrt_cuda.h (libmrt_cuda.so, built by
``python -m mobileraytracer_b200.build``).  This module is a thin Python binding of that ABI for
tests and benchmarks; it has no compute of its own and no CPU fallback: every call goes to the
device and raises MrtError when the library or the GPU is unavailable.

    ctx = Context(0)
    scn = Scene(ctx, scenes.triangle_soup(1_000_000))
    scn.build(capi.MRT_ACCEL_BVH)
    bitmap, accum, stats = scn.render(camera, capi.render_opts(width=1920, height=1080))
"""
from __future__ import annotations

import ctypes
import weakref

import numpy as np

from . import capi

__all__ = ["Context", "Scene", "Batch", "Arena", "MrtError", "capi"]

RAY_DTYPE = np.dtype([("origin", np.float32, 3), ("direction", np.float32, 3), ("depth", np.int32),
                      ("exclude", np.uint32)])
HIT_DTYPE = np.dtype([("t", np.float32), ("id", np.uint32)])


class MrtError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{capi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _is_torch_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and bool(getattr(x, "is_cuda"))


def _after_torch(ctx, *tensors):
    """The library works on its own streams: make the context's stream wait for the work torch has
    queued on its current stream (e.g. the zeroing or upload of a device buffer passed in)."""
    if any(_is_torch_cuda(t) for t in tensors if t is not None):
        import torch
        torch.cuda.ExternalStream(ctx.stream).wait_stream(torch.cuda.current_stream())


def _ptr(x):
    """(pointer, mem flag) for a numpy array (host) or a CUDA torch tensor (device)."""
    if _is_torch_cuda(x):
        return ctypes.c_void_p(x.data_ptr()), capi.MRT_MEM_DEVICE
    a = np.ascontiguousarray(x)
    return ctypes.c_void_p(a.ctypes.data), capi.MRT_MEM_HOST


class Context:
    """One CUDA device and stream (MrtContext)."""

    def __init__(self, device: int = 0):
        self.lib = capi.load()
        h = ctypes.c_void_p()
        st = self.lib.mrt_context_create(device, ctypes.byref(h))
        if st != capi.MRT_OK:
            raise MrtError(st, f"mrt_context_create(device={device}) failed")
        self.h = h
        self.device = device
        self._scenes = weakref.WeakSet()
        self._batches = weakref.WeakSet()

    def set_arena(self, arena: "Arena | None"):
        """Later device allocations of this context (scenes, their build scratch) come from `arena`."""
        self.check(self.lib.mrt_context_set_arena(self.h, arena.h if arena is not None else None), "set_arena")
        self._arena = arena

    def check(self, st: int, what: str):
        if st != capi.MRT_OK:
            raise MrtError(st, f"{what}: {self.lib.mrt_context_error(self.h).decode(errors='replace')}")

    def synchronize(self):
        self.check(self.lib.mrt_context_synchronize(self.h), "synchronize")

    @property
    def stream(self) -> int:
        return int(self.lib.mrt_context_stream(self.h) or 0)

    def close(self):
        """Destroys the context; batches and scenes still open on it are destroyed first."""
        if getattr(self, "h", None):
            for b in list(getattr(self, "_batches", ())):
                b.close()
            for s in list(getattr(self, "_scenes", ())):
                s.close()
            self.lib.mrt_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """A device-resident scene (MrtScene) with its accelerator."""

    def __init__(self, ctx: Context, scene):
        self.ctx = ctx
        self.lib = ctx.lib
        self.host = scene
        self._desc = scene.desc()
        h = ctypes.c_void_p()
        if not ctx.h:
            raise MrtError(capi.MRT_ERR_STATE, "context is closed")
        ctx.check(self.lib.mrt_scene_create(ctx.h, ctypes.byref(self._desc), ctypes.byref(h)), "mrt_scene_create")
        self.h = h
        ctx._scenes.add(self)

    def build(self, accelerator: int = capi.MRT_ACCEL_BVH, bvh_mode: int = capi.MRT_BVH_FAST, grid_size: int = 0,
              grid_index: int = capi.MRT_GRID_INDEX_REFERENCE, camera_position=None, camera=None):
        """Shader::initializeAccelerators.  Grid bounds include `camera` (its getAABB), else the point
        `camera_position`, else the scene's own camera."""
        o = capi.MrtAccelOpts()
        o.accelerator, o.bvh_mode, o.grid_size, o.grid_index = accelerator, bvh_mode, grid_size, grid_index
        if camera is None and camera_position is None and self.host.camera is not None:
            camera = self.host.camera
        if camera_position is None:
            camera_position = list(camera.position) if camera is not None else [0.0, 0.0, 0.0]
        o.camera_position[:] = camera_position
        if camera is not None:
            self._build_camera = camera
            o.camera = ctypes.pointer(camera)
        self.ctx.check(self.lib.mrt_scene_build(self.h, ctypes.byref(o)), "mrt_scene_build")
        return self

    def move_to(self, ctx: Context):
        """Hand the scene to another context on the same device (mrt_scene_move)."""
        ctx.check(self.lib.mrt_scene_move(self.h, ctx.h), "mrt_scene_move")
        self.ctx._scenes.discard(self)
        self.ctx = ctx
        ctx._scenes.add(self)
        return self

    def device_bytes(self) -> int:
        return int(self.lib.mrt_scene_device_bytes(self.h))

    def accel_info(self):
        n, r, g = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int32()
        self.lib.mrt_scene_accel_info(self.h, ctypes.byref(n), ctypes.byref(r), ctypes.byref(g))
        return {"nodes": n.value, "refs": r.value, "grid_size": g.value}

    def trace_closest(self, rays, hits=None):
        n = len(rays)
        if hits is None:
            if _is_torch_cuda(rays):
                import torch
                hits = torch.empty((n, 2), dtype=torch.int32, device=rays.device)
            else:
                hits = np.zeros(n, HIT_DTYPE)
        rp, mem = _ptr(rays)
        hp, mem2 = _ptr(hits)
        assert mem == mem2, "rays and hits must both be host or both be device buffers"
        _after_torch(self.ctx, rays, hits)
        self.ctx.check(self.lib.mrt_trace_closest(self.h, rp, n, hp, mem), "mrt_trace_closest")
        return hits

    def trace_any(self, rays, dist, occluded=None):
        n = len(rays)
        if occluded is None:
            if _is_torch_cuda(rays):
                import torch
                occluded = torch.empty(n, dtype=torch.uint8, device=rays.device)
            else:
                occluded = np.zeros(n, np.uint8)
        rp, mem = _ptr(rays)
        dp, _ = _ptr(dist if _is_torch_cuda(dist) else np.ascontiguousarray(dist, np.float32))
        op, _ = _ptr(occluded)
        _after_torch(self.ctx, rays, dist, occluded)
        self.ctx.check(self.lib.mrt_trace_any(self.h, rp, dp, n, op, mem), "mrt_trace_any")
        return occluded

    def trace_counts(self, rays):
        n = len(rays)
        nodes = np.zeros(n, np.uint32)
        tris = np.zeros(n, np.uint32)
        rp, mem = _ptr(rays)
        self.ctx.check(self.lib.mrt_trace_closest_counts(self.h, rp, n, ctypes.c_void_p(nodes.ctypes.data),
                                                         ctypes.c_void_p(tris.ctypes.data), capi.MRT_MEM_HOST),
                       "mrt_trace_closest_counts")
        return nodes, tris

    def render(self, camera, opts, bitmap=None, accum=None, stride_bytes: int | None = None):
        """One Renderer::renderFrame.  numpy buffers -> host path (copies inside the call);
        CUDA tensors -> device path.  Returns (bitmap, accum, MrtRenderStats)."""
        w, h = opts.width, opts.height
        if bitmap is None:
            bitmap = np.zeros((h, w), np.uint32)
        if stride_bytes is None:
            stride_bytes = w * 4
        bp, mem = _ptr(bitmap)
        ap = None
        if accum is not None:
            ap, mem2 = _ptr(accum)
            assert mem == mem2
        stats = capi.MrtRenderStats()
        _after_torch(self.ctx, bitmap, accum)
        self.ctx.check(self.lib.mrt_render(self.h, ctypes.byref(camera), ctypes.byref(opts), bp, stride_bytes, ap, mem,
                                           ctypes.byref(stats)), "mrt_render")
        return bitmap, accum, stats

    def raster_preview(self, camera, width: int, height: int, bitmap=None, stride_bytes: int | None = None):
        """The Android front end's raster preview of the scene's triangles (MainRenderer.copyFrame).
        numpy buffer -> host path; CUDA tensor -> device path.  Returns (bitmap, MrtRasterStats)."""
        if bitmap is None:
            bitmap = np.zeros((height, width), np.uint32)
        if stride_bytes is None:
            stride_bytes = width * 4
        bp, mem = _ptr(bitmap)
        stats = capi.MrtRasterStats()
        _after_torch(self.ctx, bitmap, None)
        self.ctx.check(self.lib.mrt_raster_preview(self.h, ctypes.byref(camera), width, height, bp, stride_bytes, mem,
                                                   ctypes.byref(stats)), "mrt_raster_preview")
        return bitmap, stats

    def stop(self):
        self.lib.mrt_render_stop(self.h)

    def progress(self) -> int:
        return int(self.lib.mrt_render_progress(self.h))

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h:   # a closed context already destroyed its scenes
                self.lib.mrt_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many renders as one stream of waves over a common ray pool (MrtBatch).

    Jobs are (scene, camera, options, device bitmap, device sums); each ends bit for bit as
    Scene.render with the same arguments on device buffers would leave it.  Scenes and buffers of a
    job must stay alive until the job is reported done."""

    def __init__(self, ctx: Context, wave_roots: int = 0, block_threads: int = 0, blocks_per_sm: int = 0,
                 max_jobs: int = 0, max_depth: int = 0, max_spl: int = 0, graph: bool = True,
                 max_wave_roots: int = 0, policy: int = capi.MRT_BATCH_SMALLEST_FIRST, pipelines: int = 0,
                 kernel: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        o = capi.MrtBatchOpts()
        o.wave_roots, o.block_threads, o.blocks_per_sm = wave_roots, block_threads, blocks_per_sm
        o.max_jobs, o.max_depth, o.max_spl = max_jobs, max_depth, max_spl
        o.no_graph = 0 if graph else 1
        o.max_wave_roots = max_wave_roots
        o.policy = policy
        o.pipelines = pipelines
        o.kernel = kernel
        h = ctypes.c_void_p()
        ctx.check(self.lib.mrt_batch_create(ctx.h, ctypes.byref(o), ctypes.byref(h)), "mrt_batch_create")
        self.h = h
        self._keep = {}
        ctx._batches.add(self)

    def submit(self, scene: Scene, camera, opts, bitmap, accum=None, stride_bytes: int | None = None) -> int:
        """Queue one render; bitmap (and accum) are CUDA tensors.  Returns the job id."""
        if not _is_torch_cuda(bitmap) or (accum is not None and not _is_torch_cuda(accum)):
            raise MrtError(capi.MRT_ERR_ARG, "Batch.submit takes device (CUDA tensor) buffers")
        j = capi.MrtBatchJob()
        j.scene = scene.h.value
        j.camera = camera
        j.opts = opts
        j.bitmap = bitmap.data_ptr()
        j.stride_bytes = opts.width * 4 if stride_bytes is None else stride_bytes
        j.accum = accum.data_ptr() if accum is not None else None
        jid = ctypes.c_uint64()
        _after_torch(self.ctx, bitmap, accum)
        self.ctx.check(self.lib.mrt_batch_submit(self.h, ctypes.byref(j), ctypes.byref(jid)), "mrt_batch_submit")
        self._keep[jid.value] = (scene, bitmap, accum)
        return jid.value

    def step(self, max_waves: int = 1) -> int:
        n = ctypes.c_uint32()
        self.ctx.check(self.lib.mrt_batch_step(self.h, max_waves, ctypes.byref(n)), "mrt_batch_step")
        return n.value

    def completed(self) -> list[int]:
        """Ids of the jobs finished since the last call."""
        out = []
        buf = (ctypes.c_uint64 * 256)()
        while True:
            n = ctypes.c_uint32()
            self.ctx.check(self.lib.mrt_batch_completed(self.h, buf, 256, ctypes.byref(n)), "mrt_batch_completed")
            out += list(buf[:n.value])
            if n.value < 256:
                break
        for jid in out:
            self._keep.pop(jid, None)
        return out

    def run(self):
        """Render every submitted job to completion."""
        self.ctx.check(self.lib.mrt_batch_run(self.h), "mrt_batch_run")

    def stats(self) -> capi.MrtBatchStats:
        s = capi.MrtBatchStats()
        self.ctx.check(self.lib.mrt_batch_stats(self.h, ctypes.byref(s)), "mrt_batch_stats")
        return s

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h:
                self.lib.mrt_batch_destroy(self.h)
            self.h = None
            self._keep = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Arena:
    """One device allocation that scenes of the contexts using it are carved from (MrtArena)."""

    def __init__(self, device: int, nbytes: int):
        self.lib = capi.load()
        h = ctypes.c_void_p()
        st = self.lib.mrt_arena_create(device, int(nbytes), ctypes.byref(h))
        if st != capi.MRT_OK:
            raise MrtError(st, f"mrt_arena_create({nbytes} bytes on device {device}) failed")
        self.h = h
        self.device = device

    def stats(self) -> dict:
        v = [ctypes.c_uint64() for _ in range(4)]
        self.lib.mrt_arena_stats(self.h, *[ctypes.byref(x) for x in v])
        return {"capacity": v[0].value, "used": v[1].value, "peak": v[2].value, "largest_free": v[3].value}

    def close(self):
        """Frees the arena; raises while scenes carved from it are alive."""
        if getattr(self, "h", None):
            st = self.lib.mrt_arena_destroy(self.h)
            if st != capi.MRT_OK:
                raise MrtError(st, "mrt_arena_destroy: buffers carved from the arena are still alive")
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
