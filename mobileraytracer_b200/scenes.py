"""Procedural scenes for the benchmark configurations, as flat arrays in the MrtSceneDesc layout.

Every generator is deterministic for a given seed: uniforms come from splitmix64 (Steele, Lea and
Flood, "Fast splittable pseudorandom number generators", 2014) evaluated with numpy uint64
arithmetic, so the same integers come out on every machine; geometry is computed in float64 and
rounded to float32 once at the end.

The reference has no procedural scenes (its four scenes are hard-coded in app/Scenes/Scenes.cpp and
its benchmark models are OBJ files that are not distributed); these are the synthetic stand-ins for
the workloads the reference is measured on:
  cornell_box()       Whitted, 256x256: 5 walls (10 tris), 2 boxes (24 tris), 1 mirror sphere,
                      2 area-light triangles of emission 15.
  triangle_soup(n)    NoShadows stress: n random equilateral triangles, 1 point light.
  heightfield()       PathTracer: 512x512 fBm terrain (524,288 tris), 4 area-light quads.
  batched_jobs()      256 soups of log-uniform size/resolution for the batched renderer.
  glass_room()        planes + spheres (mirror, glass) + triangles + area lights, to exercise every
                      primitive type and the reflect / refract branches.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import capi

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """n consecutive splitmix64 outputs for (seed, stream) as uint64."""
    gamma = np.uint64(0x9E3779B97F4A7C15)
    start = np.uint64((seed * 0x632BE59BD9B4E019 + stream * 0xD1B54A32D192ED03 + 0x1234567) & 0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        z = start + gamma * (np.arange(1, n + 1, dtype=np.uint64))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """n float64 uniforms in [0, 1) from the top 53 bits of splitmix64."""
    return (splitmix64(seed, n, stream) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _material(le=(0, 0, 0), kd=(0, 0, 0), ks=(0, 0, 0), kt=(0, 0, 0), ior=1.0) -> capi.MrtMaterial:
    m = capi.MrtMaterial()
    m.le[:] = le
    m.kd[:] = kd
    m.ks[:] = ks
    m.kt[:] = kt
    m.ior = ior
    return m


@dataclass
class Scene:
    """Host-side scene arrays (the Scene of app/MobileRT/Scene.hpp:23-27 as flat buffers)."""

    tri_abc: np.ndarray = field(default_factory=lambda: np.zeros((0, 9), np.float32))
    tri_normals: np.ndarray | None = None
    tri_colors: np.ndarray | None = None
    tri_material: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    spheres: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.float32))
    sphere_material: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    planes: np.ndarray = field(default_factory=lambda: np.zeros((0, 6), np.float32))
    plane_material: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    materials: list = field(default_factory=list)
    lights: list = field(default_factory=list)
    camera: capi.MrtCamera | None = None

    def __post_init__(self):
        self._keep = []

    @property
    def n_triangles(self) -> int:
        return int(self.tri_abc.shape[0])

    def desc(self) -> capi.MrtSceneDesc:
        """MrtSceneDesc pointing at this object's arrays (valid while the object lives)."""
        d = capi.MrtSceneDesc()
        self._keep = []

        def ptr(a, ctype):
            if a is None:
                return None
            a = np.ascontiguousarray(a)
            self._keep.append(a)
            return a.ctypes.data_as(ctypes.POINTER(ctype))

        d.n_triangles = self.n_triangles
        d.tri_abc = ptr(self.tri_abc.astype(np.float32, copy=False), ctypes.c_float)
        d.tri_normals = ptr(None if self.tri_normals is None else self.tri_normals.astype(np.float32, copy=False), ctypes.c_float)
        d.tri_colors = ptr(None if self.tri_colors is None else self.tri_colors.astype(np.float32, copy=False), ctypes.c_float)
        d.tri_material = ptr(self.tri_material.astype(np.int32, copy=False), ctypes.c_int32)
        d.n_spheres = int(self.spheres.shape[0])
        d.sphere_center_radius = ptr(self.spheres.astype(np.float32, copy=False), ctypes.c_float)
        d.sphere_material = ptr(self.sphere_material.astype(np.int32, copy=False), ctypes.c_int32)
        d.n_planes = int(self.planes.shape[0])
        d.plane_point_normal = ptr(self.planes.astype(np.float32, copy=False), ctypes.c_float)
        d.plane_material = ptr(self.plane_material.astype(np.int32, copy=False), ctypes.c_int32)
        mats = (capi.MrtMaterial * max(1, len(self.materials)))(*self.materials)
        lights = (capi.MrtLightDesc * max(1, len(self.lights)))(*self.lights)
        self._keep += [mats, lights]
        d.n_materials = len(self.materials)
        d.materials = ctypes.cast(mats, ctypes.POINTER(capi.MrtMaterial))
        d.n_lights = len(self.lights)
        d.lights = ctypes.cast(lights, ctypes.POINTER(capi.MrtLightDesc))
        return d

    def device_footprint_estimate(self) -> int:
        """Bytes the scene needs on the device (geometry + fast BVH), for admission decisions."""
        n = self.n_triangles
        return 48 * n + 76 * n + 64 * n + 4 * n + 4096


def point_light(pos, le=(0.9, 0.9, 0.9)) -> capi.MrtLightDesc:
    l = capi.MrtLightDesc()
    l.kind = capi.MRT_LIGHT_POINT
    l.p0[:] = pos
    l.radiance = _material(le=le)
    return l


def area_light(a, b, c, le) -> capi.MrtLightDesc:
    l = capi.MrtLightDesc()
    l.kind = capi.MRT_LIGHT_AREA
    l.p0[:] = a
    l.p1[:] = b
    l.p2[:] = c
    l.radiance = _material(le=le)
    return l


def camera(position, look_at, up=(0.0, 1.0, 0.0), fov_h=45.0, fov_v=45.0) -> capi.MrtCamera:
    c = capi.MrtCamera()
    c.kind = capi.MRT_CAMERA_PERSPECTIVE
    c.position[:] = position
    c.look_at[:] = look_at
    c.up[:] = up
    c.fov_h_deg = fov_h
    c.fov_v_deg = fov_v
    return c


def orthographic(position, look_at, up=(0.0, 1.0, 0.0), size_h=2.0, size_v=2.0) -> capi.MrtCamera:
    """Components::Orthographic(position, lookAt, up, sizeH, sizeV) (Orthographic.cpp:12-17)."""
    c = camera(position, look_at, up, size_h, size_v)
    c.kind = capi.MRT_CAMERA_ORTHOGRAPHIC
    return c


def cli_camera(width: int, height: int) -> capi.MrtCamera:
    """The Linux CLI's default camera (c_wrapper.cpp:56-67): eye (0,0,-3.4) looking at +z,
    45 degrees scaled by the aspect ratio on the wider axis (float32 products, as there)."""
    ratio = np.float32(width) / np.float32(height)
    hf = np.float32(45.0) * max(ratio, np.float32(1.0))
    vf = np.float32(45.0) * max(np.float32(1.0) / ratio, np.float32(1.0))
    return camera((0.0, 0.0, -3.4), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), float(hf), float(vf))


def _oriented_tri(a, b, c, normal):
    """Order (a, b, c) so the reference's computed normal, normalize(cross(C - A, B - A)),
    points along `normal` (Triangle.cpp 4-argument constructor)."""
    a, b, c = (np.asarray(v, np.float64) for v in (a, b, c))
    n = np.cross(c - a, b - a)
    if np.dot(n, normal) < 0:
        b, c = c, b
    return np.concatenate([a, b, c])


def _quad(p0, p1, p2, p3, normal):
    return [_oriented_tri(p0, p1, p2, normal), _oriented_tri(p0, p2, p3, normal)]


def _box(lo, hi):
    """12 outward-facing triangles of an axis-aligned box."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = lambda x, y, z: (x, y, z)
    faces = [
        ((v(x0, y0, z0), v(x1, y0, z0), v(x1, y0, z1), v(x0, y0, z1)), (0, -1, 0)),
        ((v(x0, y1, z0), v(x1, y1, z0), v(x1, y1, z1), v(x0, y1, z1)), (0, 1, 0)),
        ((v(x0, y0, z0), v(x1, y0, z0), v(x1, y1, z0), v(x0, y1, z0)), (0, 0, -1)),
        ((v(x0, y0, z1), v(x1, y0, z1), v(x1, y1, z1), v(x0, y1, z1)), (0, 0, 1)),
        ((v(x0, y0, z0), v(x0, y1, z0), v(x0, y1, z1), v(x0, y0, z1)), (-1, 0, 0)),
        ((v(x1, y0, z0), v(x1, y1, z0), v(x1, y1, z1), v(x1, y0, z1)), (1, 0, 0)),
    ]
    tris = []
    for quad, n in faces:
        tris += _quad(*quad, np.asarray(n, np.float64))
    return tris


def cornell_box() -> Scene:
    """Unit Cornell box centred at the origin, open towards the camera (-z)."""
    white, red, green = 0, 1, 2
    mats = [
        _material(kd=(0.73, 0.73, 0.73)),
        _material(kd=(0.63, 0.065, 0.05)),
        _material(kd=(0.14, 0.45, 0.09)),
        _material(ks=(0.9, 0.9, 0.9)),   # mirror: Kd 0, Ks 0.9
    ]
    h = 0.5
    tris, tmat = [], []

    def add(ts, m):
        tris.extend(ts)
        tmat.extend([m] * len(ts))

    add(_quad((-h, -h, -h), (h, -h, -h), (h, -h, h), (-h, -h, h), np.array([0, 1, 0.0])), white)   # floor
    add(_quad((-h, h, -h), (h, h, -h), (h, h, h), (-h, h, h), np.array([0, -1, 0.0])), white)      # ceiling
    add(_quad((-h, -h, h), (h, -h, h), (h, h, h), (-h, h, h), np.array([0, 0, -1.0])), white)      # back
    add(_quad((-h, -h, -h), (-h, h, -h), (-h, h, h), (-h, -h, h), np.array([1, 0, 0.0])), red)     # left
    add(_quad((h, -h, -h), (h, h, -h), (h, h, h), (h, -h, h), np.array([-1, 0, 0.0])), green)      # right
    add(_box((-0.38, -0.5, 0.02), (-0.08, 0.12, 0.32)), white)   # tall box
    add(_box((0.05, -0.5, -0.3), (0.33, -0.22, -0.02)), white)   # short box
    s = Scene()
    s.tri_abc = np.asarray(tris, np.float32)
    s.tri_material = np.asarray(tmat, np.int32)
    s.materials = mats
    s.spheres = np.asarray([[0.19, -0.07, -0.16, 0.15]], np.float32)   # mirror sphere on the short box
    s.sphere_material = np.asarray([3], np.int32)
    y = 0.499
    s.lights = [
        area_light((-0.12, y, -0.12), (0.12, y, -0.12), (0.12, y, 0.12), (15.0, 15.0, 15.0)),
        area_light((-0.12, y, -0.12), (0.12, y, 0.12), (-0.12, y, 0.12), (15.0, 15.0, 15.0)),
    ]
    s.camera = camera((0.0, 0.0, -1.7), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 45.0)
    return s


def _soup_geometry(n: int, seed: int) -> np.ndarray:
    """n equilateral triangles: centroid ~ U[-1,1]^3, side ~ lognormal(ln 0.005, 0.5),
    orientation ~ uniform random rotation (Shoemake's unit quaternion)."""
    u = uniform(seed, 8 * n).reshape(n, 8)
    centre = 2.0 * u[:, 0:3] - 1.0
    z = np.sqrt(-2.0 * np.log1p(-u[:, 3])) * np.cos(2.0 * math.pi * u[:, 4])   # Box-Muller
    side = np.exp(math.log(0.005) + 0.5 * z)
    u1, u2, u3 = u[:, 5], u[:, 6], u[:, 7]
    qx = np.sqrt(1.0 - u1) * np.sin(2 * math.pi * u2)
    qy = np.sqrt(1.0 - u1) * np.cos(2 * math.pi * u2)
    qz = np.sqrt(u1) * np.sin(2 * math.pi * u3)
    qw = np.sqrt(u1) * np.cos(2 * math.pi * u3)
    rot = np.stack([
        np.stack([1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)], -1),
        np.stack([2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)], -1),
        np.stack([2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)], -1),
    ], -2)   # (n, 3, 3)
    ang = np.array([0.5 * math.pi, 0.5 * math.pi + 2 * math.pi / 3, 0.5 * math.pi + 4 * math.pi / 3])
    canon = np.stack([np.cos(ang), np.sin(ang), np.zeros(3)], -1) / math.sqrt(3.0)   # unit side, centroid 0
    verts = np.einsum("nij,kj->nki", rot, canon) * side[:, None, None] + centre[:, None, :]
    return verts.reshape(n, 9).astype(np.float32)


def triangle_soup(n: int = 1_000_000, seed: int = 0, width: int = 1920, height: int = 1080) -> Scene:
    """Triangle soup with one white diffuse material and one point light."""
    s = Scene()
    s.tri_abc = _soup_geometry(n, seed)
    s.tri_material = np.zeros(n, np.int32)
    s.materials = [_material(kd=(0.8, 0.8, 0.8))]
    s.lights = [point_light((0.0, 2.5, -2.5), (0.9, 0.9, 0.9))]
    s.camera = cli_camera(width, height)
    return s


def _value_noise(x: np.ndarray, z: np.ndarray, seed: int, octave: int) -> np.ndarray:
    ix, iz = np.floor(x).astype(np.int64), np.floor(z).astype(np.int64)
    fx, fz = x - ix, z - iz

    def lattice(i, k):
        h = (i * 0x9E3779B1 + k * 0x85EBCA77 + seed * 0xC2B2AE3D + octave * 0x27D4EB2F) & 0xFFFFFFFF
        h = h.astype(np.uint64)
        with np.errstate(over="ignore"):
            h = (h ^ (h >> np.uint64(15))) * np.uint64(0x2C1B3C6D) & np.uint64(0xFFFFFFFF)
            h = (h ^ (h >> np.uint64(12))) * np.uint64(0x297A2D39) & np.uint64(0xFFFFFFFF)
            h = h ^ (h >> np.uint64(15))
        return (h & np.uint64(0xFFFFFF)).astype(np.float64) / 16777216.0

    sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
    a, b = lattice(ix, iz), lattice(ix + 1, iz)
    c, d = lattice(ix, iz + 1), lattice(ix + 1, iz + 1)
    return (a * (1 - sx) + b * sx) * (1 - sz) + (c * (1 - sx) + d * sx) * sz


def heightfield(cells: int = 512, seed: int = 1, octaves: int = 6, gain: float = 0.5, lacunarity: float = 2.0,
                amplitude: float = 0.35, width: int = 1024, height: int = 1024) -> Scene:
    """fBm value-noise terrain over [-1,1]^2 (2*cells^2 triangles), grey albedo per
    triangle ~ U[0.2, 0.8] carried in the triangle colours (material -1, NoShadows.cpp:35-36
    kD = primitive colour), 4 area-light quads (8 AreaLight triangles) of emission 10."""
    g = np.linspace(-1.0, 1.0, cells + 1)
    X, Z = np.meshgrid(g, g, indexing="ij")
    H = np.zeros_like(X)
    amp, freq = 0.5, 4.0
    for o in range(octaves):
        H += amp * (_value_noise((X + 1) * freq, (Z + 1) * freq, seed, o) - 0.5)
        amp *= gain
        freq *= lacunarity
    H *= 2.0 * amplitude
    V = np.stack([X, H, Z], -1)
    v00, v10 = V[:-1, :-1], V[1:, :-1]
    v01, v11 = V[:-1, 1:], V[1:, 1:]
    t1 = np.concatenate([v00, v10, v11], -1).reshape(-1, 9)
    t2 = np.concatenate([v00, v11, v01], -1).reshape(-1, 9)
    tris = np.stack([t1, t2], 1).reshape(-1, 9)   # cell-major, 2 per cell
    n = tris.shape[0]
    albedo = 0.2 + 0.6 * uniform(seed, n, stream=7)
    s = Scene()
    s.tri_abc = tris.astype(np.float32)
    s.tri_colors = np.repeat(albedo[:, None], 9, 1).astype(np.float32)
    s.tri_material = np.full(n, -1, np.int32)
    s.lights = _quad_lights(10.0)
    s.camera = camera((0.0, 1.25, -2.15), (0.0, 0.0, 0.05), (0.0, 1.0, 0.0), 45.0 * max(width / height, 1.0),
                      45.0 * max(height / width, 1.0))
    return s


def _quad_lights(le: float):
    lights = []
    y, r = 1.3, 0.15
    for cx, cz in ((-0.5, -0.5), (0.5, -0.5), (-0.5, 0.5), (0.5, 0.5)):
        a, b, c, d = (cx - r, y, cz - r), (cx + r, y, cz - r), (cx + r, y, cz + r), (cx - r, y, cz + r)
        lights.append(area_light(a, b, c, (le, le, le)))
        lights.append(area_light(a, c, d, (le, le, le)))
    return lights


@dataclass
class Job:
    """One render request of the batched / served workloads."""

    index: int
    n_triangles: int
    side: int
    spp: int
    seed: int

    def scene(self) -> Scene:
        s = Scene()
        s.tri_abc = _soup_geometry(self.n_triangles, self.seed)
        s.tri_material = np.zeros(self.n_triangles, np.int32)
        s.materials = [_material(kd=(0.8, 0.8, 0.8))]
        s.lights = _quad_lights(10.0)
        s.camera = cli_camera(self.side, self.side)
        return s


def batched_jobs(count: int = 256, n_min: float = 1e3, n_max: float = 2e6, side_min: int = 128,
                 side_max: int = 1024, spps=(1, 4, 16, 64)) -> list[Job]:
    """Batched job list: job i uses seed i; N ~ log-uniform[n_min, n_max]; image side
    ~ log-uniform[side_min, side_max] rounded down to a multiple of 16 (the reference's block
    schedule covers exactly such images, Renderer.cpp:20-21); spp uniform over `spps`."""
    jobs = []
    for i in range(count):
        u = uniform(i, 3, stream=11)
        n = int(round(math.exp(math.log(n_min) + u[0] * (math.log(n_max) - math.log(n_min)))))
        side = int(math.exp(math.log(side_min) + u[1] * (math.log(side_max) - math.log(side_min))))
        side = max(side_min, side - side % 16)
        spp = int(spps[min(len(spps) - 1, int(u[2] * len(spps)))])
        jobs.append(Job(i, n, side, spp, i))
    return jobs


def load_obj(obj_path: str, mtl_path: str | None = None, camera: capi.MrtCamera | None = None) -> Scene:
    """A scene from a Wavefront OBJ (and the MTL file named here) through the library's loader,
    mrt_obj_load (the reference's OBJLoader conventions); the arrays are copied into numpy."""
    lib = capi.load()
    h = ctypes.c_void_p()
    d = capi.MrtSceneDesc()
    err = ctypes.create_string_buffer(512)
    st = lib.mrt_obj_load(obj_path.encode(), mtl_path.encode() if mtl_path else None, ctypes.byref(h),
                          ctypes.byref(d), err, len(err))
    if st != capi.MRT_OK:
        from . import MrtError
        raise MrtError(st, err.value.decode(errors="replace"))
    try:
        n = d.n_triangles
        s = Scene()

        def arr(ptr, count, dtype):
            if count == 0 or not ptr:
                return np.zeros(count, dtype)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype).copy()

        s.tri_abc = arr(d.tri_abc, 9 * n, np.float32).reshape(n, 9)
        s.tri_normals = arr(d.tri_normals, 9 * n, np.float32).reshape(n, 9)
        s.tri_colors = arr(d.tri_colors, 9 * n, np.float32).reshape(n, 9)
        s.tri_material = arr(d.tri_material, n, np.int32)
        s.materials = [capi.MrtMaterial.from_buffer_copy(d.materials[i]) for i in range(d.n_materials)]
        s.lights = [capi.MrtLightDesc.from_buffer_copy(d.lights[i]) for i in range(d.n_lights)]
        s.camera = camera
        return s
    finally:
        lib.mrt_obj_free(h)


def glass_room() -> Scene:
    """Every primitive type and material branch: 6 planes (a closed room), a mirror sphere, a glass
    sphere (ior 1.9), a diffuse+specular sphere, two coloured triangles with given normals and
    colours, one triangle without material (colour shading), two area lights."""
    mats = [
        _material(kd=(0.7, 0.7, 0.7)),                       # 0 white
        _material(kd=(0.9, 0.0, 0.0)),                       # 1 red
        _material(kd=(0.0, 0.0, 0.9)),                       # 2 blue
        _material(ks=(0.9, 0.9, 0.9)),                       # 3 mirror
        _material(kt=(0.9, 0.9, 0.9), ior=1.9),              # 4 glass
        _material(kd=(0.2, 0.6, 0.2), ks=(0.5, 0.5, 0.5)),   # 5 diffuse + specular
        _material(kd=(0.9, 0.9, 0.0)),                       # 6 yellow
    ]
    s = Scene()
    s.materials = mats
    s.planes = np.asarray([
        [0, -1, 0, 0, 1, 0], [0, 1, 0, 0, -1, 0], [-1, 0, 0, 1, 0, 0],
        [1, 0, 0, -1, 0, 0], [0, 0, 1, 0, 0, -1], [0, 0, -4, 0, 0, 1],
    ], np.float32)
    s.plane_material = np.asarray([0, 0, 1, 2, 0, 0], np.int32)
    s.spheres = np.asarray([[0.45, -0.65, 0.4, 0.35], [-0.4, -0.3, 0.0, 0.35], [0.1, 0.3, 0.6, 0.2]], np.float32)
    s.sphere_material = np.asarray([3, 4, 5], np.int32)
    s.tri_abc = np.asarray([
        [0.5, -0.5, 0.99, 0.5, 0.5, 1.001, -0.5, -0.5, 0.99],
        [-0.6, 0.55, 0.9, -0.6, -0.2, 0.95, 0.2, 0.55, 0.9],
        [0.6, -0.9, -0.2, 0.9, -0.9, 0.3, 0.6, -0.3, 0.3],
    ], np.float32)
    nrm = np.asarray([[0, 0, -1] * 3, [-1, 1, -1, -1, -1, -1, 1, 1, -1], [0, 0, -1] * 3], np.float32)
    s.tri_normals = nrm
    s.tri_colors = np.asarray([[1, 0, 0, 0, 1, 0, 0, 0, 1], [1, 1, 1] * 3, [0.3, 0.8, 0.3] * 3], np.float32)
    s.tri_material = np.asarray([6, 3, -1], np.int32)
    s.lights = [
        area_light((-0.25, 0.99, -0.25), (0.25, 0.99, -0.25), (0.25, 0.99, 0.25), (0.9, 0.9, 0.9)),
        area_light((0.25, 0.99, 0.25), (-0.25, 0.99, 0.25), (-0.25, 0.99, -0.25), (0.9, 0.9, 0.9)),
    ]
    s.camera = camera((0.0, 0.0, -3.4), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 45.0)
    return s
