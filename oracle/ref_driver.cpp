// ref_driver.cpp - C entry points around the reference's own compiled classes.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product): oracle/Makefile compiles this file
// together with an unmodified copy of the reference render sources (one conformance line patched,
// see the Makefile) into oracle/_ref/liboracle_ref.so.  Tests, the smoke check and the CPU baseline
// of bench.py call it through ctypes to obtain the reference's own answers:
//   * shape/box known-answer values     Triangle.cpp, Sphere.cpp, Plane.cpp, AABB.cpp
//   * closest-hit ids / any-hit flags   Shader::rayTrace / Shader::shadowTrace (Shader.cpp:124-187)
//                                       through the reference's own accelerators
//   * whole frames                      Renderer::renderFrame (Renderer.cpp:31-116)
//   * OBJ scenes                        OBJLoader::process + OBJLoader::fillScene (OBJLoader.cpp:21-248)
//                                       on a parse staged by the caller (tinyobjloader is absent)
// Scenes arrive in the mrt_cuda.h MrtSceneDesc layout so the same arrays feed the CUDA path.
#include "../include/mrt_cuda.h"

#include "Components/Cameras/Orthographic.hpp"
#include "Components/Cameras/Perspective.hpp"
#include "Components/Lights/AreaLight.hpp"
#include "Components/ObjectLoaders/OBJLoader.hpp"
#include "Components/Lights/PointLight.hpp"
#include "Components/Samplers/Constant.hpp"
#include "Components/Samplers/HaltonSeq.hpp"
#include "Components/Samplers/MersenneTwister.hpp"
#include "Components/Samplers/Stratified.hpp"
#include "Components/Shaders/DepthMap.hpp"
#include "Components/Shaders/DiffuseMaterial.hpp"
#include "Components/Shaders/NoShadows.hpp"
#include "Components/Shaders/PathTracer.hpp"
#include "Components/Shaders/Whitted.hpp"
#include "MobileRT/Renderer.hpp"
#include "MobileRT/Scene.hpp"
#include "MobileRT/Shader.hpp"
#include "MobileRT/Utils.hpp"

#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

using ::MobileRT::AABB;
using ::MobileRT::Intersection;
using ::MobileRT::Material;
using ::MobileRT::Plane;
using ::MobileRT::Ray;
using ::MobileRT::Scene;
using ::MobileRT::Shader;
using ::MobileRT::Sphere;
using ::MobileRT::Triangle;

namespace {

::glm::vec3 v3(const float *p) { return ::glm::vec3{p[0], p[1], p[2]}; }

Material to_material(const MrtMaterial &m) {
    return Material{v3(m.kd), v3(m.ks), v3(m.kt), m.ior, v3(m.le)};
}

std::unique_ptr<::MobileRT::Sampler> make_sampler(int kind, float value, uint32_t w, uint32_t h, uint32_t spp) {
    switch (kind) {
        case MRT_SAMPLER_CONSTANT: return std::make_unique<::Components::Constant>(value);
        case MRT_SAMPLER_STRATIFIED: return std::make_unique<::Components::Stratified>(w, h, spp);
        case MRT_SAMPLER_HALTON: return std::make_unique<::Components::HaltonSeq>(w, h, spp);
        default: return std::make_unique<::Components::MersenneTwister>();
    }
}

Triangle make_triangle(const MrtSceneDesc &d, uint32_t i) {
    const float *p = d.tri_abc + 9 * i;
    const int32_t mat = d.tri_material ? d.tri_material[i] : -1;
    if (d.tri_normals != nullptr) {
        const float *n = d.tri_normals + 9 * i;
        const float zero[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const float *c = d.tri_colors ? d.tri_colors + 9 * i : zero;
        return Triangle{v3(p), v3(p + 3), v3(p + 6), mat, v3(n), v3(n + 3), v3(n + 6), v3(c), v3(c + 3), v3(c + 6)};
    }
    if (d.tri_colors != nullptr) {
        const float *c = d.tri_colors + 9 * i;
        return Triangle{v3(p), v3(p + 3), v3(p + 6), mat, v3(c), v3(c + 3), v3(c + 6)};
    }
    return Triangle{v3(p), v3(p + 3), v3(p + 6), mat};
}

Scene make_scene(const MrtSceneDesc &d, int light_sampler, float cval, uint32_t w, uint32_t h, uint32_t spp) {
    Scene scene{};
    scene.triangles_.reserve(d.n_triangles);
    for (uint32_t i = 0; i < d.n_triangles; ++i) scene.triangles_.emplace_back(make_triangle(d, i));
    for (uint32_t i = 0; i < d.n_spheres; ++i) {
        const float *s = d.sphere_center_radius + 4 * i;
        scene.spheres_.emplace_back(Sphere{v3(s), s[3], d.sphere_material ? d.sphere_material[i] : -1});
    }
    for (uint32_t i = 0; i < d.n_planes; ++i) {
        const float *p = d.plane_point_normal + 6 * i;
        scene.planes_.emplace_back(Plane{v3(p), v3(p + 3), d.plane_material ? d.plane_material[i] : -1});
    }
    for (uint32_t i = 0; i < d.n_materials; ++i) scene.materials_.emplace_back(to_material(d.materials[i]));
    for (uint32_t i = 0; i < d.n_lights; ++i) {
        const MrtLightDesc &l = d.lights[i];
        if (l.kind == MRT_LIGHT_AREA) {
            scene.lights_.emplace_back(std::make_unique<::Components::AreaLight>(
                to_material(l.radiance), make_sampler(light_sampler, cval, w, h, spp), v3(l.p0), v3(l.p1), v3(l.p2)));
        } else {
            scene.lights_.emplace_back(std::make_unique<::Components::PointLight>(to_material(l.radiance), v3(l.p0)));
        }
    }
    return scene;
}

// Shader whose shade() records the intersection instead of shading it, so Shader::rayTrace (the
// reference's own type-ordered accelerator dispatch) can be driven ray by ray.
struct HitRecord {
    bool hit;
    float length;
    const void *primitive;
    int32_t material_id;
};
thread_local HitRecord tl_record;

class IdShader final : public Shader {
public:
    IdShader(Scene &&scene, Accelerator a) : Shader{std::move(scene), 1, a} {}
    bool shade(::glm::vec3 *, const Intersection &it, const Ray &) noexcept final {
        tl_record = HitRecord{true, it.length_, it.primitive_, it.materialId_};
        return false;
    }
};

template <typename T> const T *storage(const Shader &s, int accel);
template <> const Triangle *storage<Triangle>(const Shader &s, int a) {
    return a == MRT_ACCEL_NAIVE ? s.naiveTriangles_.primitives_.data()
         : a == MRT_ACCEL_BVH ? s.bvhTriangles_.primitives_.data() : s.scene_.triangles_.data();
}
template <> const Plane *storage<Plane>(const Shader &s, int a) {
    return a == MRT_ACCEL_NAIVE ? s.naivePlanes_.primitives_.data()
         : a == MRT_ACCEL_BVH ? s.bvhPlanes_.primitives_.data() : s.scene_.planes_.data();
}
template <> const Sphere *storage<Sphere>(const Shader &s, int a) {
    return a == MRT_ACCEL_NAIVE ? s.naiveSpheres_.primitives_.data()
         : a == MRT_ACCEL_BVH ? s.bvhSpheres_.primitives_.data() : s.scene_.spheres_.data();
}

struct TraceHandle {
    std::unique_ptr<IdShader> shader;
    std::unique_ptr<::MobileRT::Camera> camera;
    int accel;
    uint32_t n_tri, n_sph, n_pln, n_lights;
};

const void *exclude_pointer(const TraceHandle &h, uint32_t id) {
    if (id == MRT_HIT_NONE) return nullptr;
    const uint32_t idx = MRT_HIT_INDEX(id);
    switch (MRT_HIT_TYPE(id)) {
        case MRT_PRIM_TRIANGLE: return idx < h.n_tri ? storage<Triangle>(*h.shader, h.accel) + idx : nullptr;
        case MRT_PRIM_PLANE: return idx < h.n_pln ? storage<Plane>(*h.shader, h.accel) + idx : nullptr;
        case MRT_PRIM_SPHERE: return nullptr;  // spheres never exclude themselves (Sphere.cpp:18-52)
        default: {
            // an area light's triangle lives inside the AreaLight object; exclusion by pointer only
            // matters for rays leaving a light, which the shaders never spawn
            return nullptr;
        }
    }
}

uint32_t identify(const TraceHandle &h, const Ray &ray, const HitRecord &r) {
    const char *p = static_cast<const char *>(r.primitive);
    if (p != nullptr) {
        const char *tb = reinterpret_cast<const char *>(storage<Triangle>(*h.shader, h.accel));
        if (h.n_tri && p >= tb && p < tb + sizeof(Triangle) * h.n_tri)
            return MRT_HIT_ID(MRT_PRIM_TRIANGLE, (p - tb) / sizeof(Triangle));
        const char *pb = reinterpret_cast<const char *>(storage<Plane>(*h.shader, h.accel));
        if (h.n_pln && p >= pb && p < pb + sizeof(Plane) * h.n_pln)
            return MRT_HIT_ID(MRT_PRIM_PLANE, (p - pb) / sizeof(Plane));
        for (uint32_t k = 0; k < h.n_lights; ++k) {
            const char *lb = reinterpret_cast<const char *>(h.shader->scene_.lights_[k].get());
            if (p >= lb && p < lb + sizeof(::Components::AreaLight)) return MRT_HIT_ID(MRT_PRIM_LIGHT, k);
        }
        return MRT_HIT_NONE - 1;  // unidentifiable: reported as a distinct value
    }
    // Sphere hits carry no primitive pointer (Sphere.cpp:48); the hit sphere is the lowest index
    // whose own intersection length equals the recorded one.
    const Sphere *sb = storage<Sphere>(*h.shader, h.accel);
    for (uint32_t k = 0; k < h.n_sph; ++k) {
        Intersection it{::MobileRT::RayLengthMax};
        if (sb[k].intersect(&it, ray) && std::memcmp(&it.length_, &r.length, sizeof(float)) == 0)
            return MRT_HIT_ID(MRT_PRIM_SPHERE, k);
    }
    return MRT_HIT_NONE - 1;
}

template <typename F> void parallel_for(uint32_t n, int threads, F &&f) {
    if (threads <= 1 || n < 64) {
        for (uint32_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<uint32_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const uint32_t b = next.fetch_add(64);
            if (b >= n) break;
            const uint32_t e = b + 64 < n ? b + 64 : n;
            for (uint32_t i = b; i < e; ++i) f(i);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

std::unique_ptr<Shader> make_shader(Scene &&scene, const MrtRenderOpts &o, int accel) {
    const auto a = static_cast<Shader::Accelerator>(accel);
    switch (o.shader) {
        case MRT_SHADER_WHITTED: return std::make_unique<::Components::Whitted>(std::move(scene), o.spl, a);
        case MRT_SHADER_PATHTRACER:
            return std::make_unique<::Components::PathTracer>(
                std::move(scene), make_sampler(o.rr_sampler, o.constant_value, o.width, o.height, o.spp), o.spl, a);
        case MRT_SHADER_DEPTHMAP:
            return std::make_unique<::Components::DepthMap>(std::move(scene), v3(o.depth_point), a);
        case MRT_SHADER_DIFFUSE: return std::make_unique<::Components::DiffuseMaterial>(std::move(scene), a);
        default: return std::make_unique<::Components::NoShadows>(std::move(scene), o.spl, a);
    }
}

std::unique_ptr<::MobileRT::Camera> make_camera(const MrtCamera &c) {
    if (c.kind == MRT_CAMERA_ORTHOGRAPHIC)
        return std::make_unique<::Components::Orthographic>(v3(c.position), v3(c.look_at), v3(c.up), c.fov_h_deg,
                                                             c.fov_v_deg);
    return std::make_unique<::Components::Perspective>(v3(c.position), v3(c.look_at), v3(c.up), c.fov_h_deg, c.fov_v_deg);
}

}  // namespace

namespace {

// ---- the staged parse behind tinyobj::LoadObj (oracle/shim/tinyobjloader/tiny_obj_loader.h) ----------
struct ObjStage {
    bool staged = false;
    ::tinyobj::attrib_t attrib;
    std::vector<::tinyobj::shape_t> shapes;
    std::vector<::tinyobj::material_t> materials;
};
ObjStage &obj_stage() {
    thread_local ObjStage st;
    return st;
}

// read access to AreaLight::triangle_ (private in the reference) through an explicit instantiation,
// which may name private members: the checker compares the light's triangle as the reference built it
template <typename Tag, typename Tag::type M>
struct Expose {
    friend typename Tag::type get(Tag) { return M; }
};
struct AreaLightTriangle {
    typedef ::MobileRT::Triangle Components::AreaLight::*type;
    friend type get(AreaLightTriangle);
};
template struct Expose<AreaLightTriangle, &Components::AreaLight::triangle_>;

}  // namespace

namespace tinyobj {
bool LoadObj(attrib_t *attrib, std::vector<shape_t> *shapes, std::vector<material_t> *materials, std::string *,
             std::string *err, std::istream *, MaterialReader *, bool) {
    ObjStage &st = obj_stage();
    if (!st.staged) {
        if (err) *err = "no staged parse";
        return false;
    }
    *attrib = st.attrib;
    *shapes = st.shapes;
    *materials = st.materials;
    return true;
}
}  // namespace tinyobj

extern "C" {

int ref_abi_version(void) { return 1; }

/* ---- shape / box known-answer entry points --------------------------------------------------- */
int ref_triangle_intersect(const float *abc, const float *normals, const float *colors, const float *o,
                           const float *d, float length, float *out_t, float *out_normal, float *out_color) {
    MrtSceneDesc desc{};
    desc.n_triangles = 1;
    desc.tri_abc = abc;
    desc.tri_normals = normals;
    desc.tri_colors = colors;
    const Triangle tri = make_triangle(desc, 0);
    Intersection it{length};
    const Ray ray{v3(d), v3(o), 1};
    const bool hit = tri.intersect(&it, ray);
    if (out_t) *out_t = it.length_;
    if (out_normal) { out_normal[0] = it.normal_[0]; out_normal[1] = it.normal_[1]; out_normal[2] = it.normal_[2]; }
    if (out_color) { out_color[0] = it.primitiveColor_[0]; out_color[1] = it.primitiveColor_[1]; out_color[2] = it.primitiveColor_[2]; }
    return hit ? 1 : 0;
}

int ref_triangle_occludes(const float *abc, const float *o, const float *d, float dist) {
    MrtSceneDesc desc{};
    desc.n_triangles = 1;
    desc.tri_abc = abc;
    const Triangle tri = make_triangle(desc, 0);
    return tri.intersect(Ray{v3(d), v3(o), 1}, dist) ? 1 : 0;
}

int ref_triangle_intersect_box(const float *abc, const float *bmin, const float *bmax) {
    MrtSceneDesc desc{};
    desc.n_triangles = 1;
    desc.tri_abc = abc;
    return make_triangle(desc, 0).intersectBox(AABB{v3(bmin), v3(bmax)}) ? 1 : 0;
}

void ref_triangle_fields(const float *abc, float *ab_ac_n) {
    MrtSceneDesc desc{};
    desc.n_triangles = 1;
    desc.tri_abc = abc;
    const Triangle t = make_triangle(desc, 0);
    const AABB b = t.getAABB();
    const float vals[15] = {t.AB_[0], t.AB_[1], t.AB_[2], t.AC_[0], t.AC_[1], t.AC_[2],
                            t.normalA_[0], t.normalA_[1], t.normalA_[2],
                            b.pointMin_[0], b.pointMin_[1], b.pointMin_[2], b.pointMax_[0], b.pointMax_[1], b.pointMax_[2]};
    std::memcpy(ab_ac_n, vals, sizeof(vals));
}

int ref_plane_intersect_box(const float *pn, const float *bmin, const float *bmax) {
    const Plane p{v3(pn), v3(pn + 3), -1};
    return p.intersectBox(AABB{v3(bmin), v3(bmax)}) ? 1 : 0;
}

float ref_plane_distance(const float *pn, const float *q) {
    const Plane p{v3(pn), v3(pn + 3), -1};
    return p.distance(v3(q));
}

int ref_plane_intersect(const float *pn, const float *o, const float *d, float length, float *out_t) {
    const Plane p{v3(pn), v3(pn + 3), -1};
    Intersection it{length};
    const bool hit = p.intersect(&it, Ray{v3(d), v3(o), 1});
    *out_t = it.length_;
    return hit ? 1 : 0;
}

void ref_plane_aabb(const float *pn, float *out6) {
    const Plane p{v3(pn), v3(pn + 3), -1};
    const AABB b = p.getAABB();
    for (int k = 0; k < 3; ++k) { out6[k] = b.pointMin_[k]; out6[3 + k] = b.pointMax_[k]; }
}

int ref_sphere_intersect(const float *cr, const float *o, const float *d, float length, float *out_t, float *out_n) {
    const Sphere s{v3(cr), cr[3], -1};
    Intersection it{length};
    const bool hit = s.intersect(&it, Ray{v3(d), v3(o), 1});
    *out_t = it.length_;
    if (out_n) { out_n[0] = it.normal_[0]; out_n[1] = it.normal_[1]; out_n[2] = it.normal_[2]; }
    return hit ? 1 : 0;
}

int ref_sphere_intersect_box(const float *cr, const float *bmin, const float *bmax) {
    const Sphere s{v3(cr), cr[3], -1};
    return s.intersectBox(AABB{v3(bmin), v3(bmax)}) ? 1 : 0;
}

int ref_aabb_intersect(const float *bmin, const float *bmax, const float *o, const float *d) {
    return ::MobileRT::intersect(AABB{v3(bmin), v3(bmax)}, Ray{v3(d), v3(o), 1}) ? 1 : 0;
}

float ref_aabb_area(const float *bmin, const float *bmax) { return AABB{v3(bmin), v3(bmax)}.getSurfaceArea(); }

float ref_halton(uint32_t index, uint32_t base) { return ::MobileRT::haltonSequence(index, base); }

uint32_t ref_incremental_avg(const float *rgb, uint32_t avg, uint32_t n) {
    return ::MobileRT::incrementalAvg(v3(rgb), avg, n);
}

void ref_camera_ray(const MrtCamera *c, float u, float v, float du, float dv, float *o6) {
    const auto cam = make_camera(*c);
    const Ray r = cam->generateRay(u, v, du, dv);
    for (int k = 0; k < 3; ++k) { o6[k] = r.origin_[k]; o6[3 + k] = r.direction_[k]; }
}

/* ---- accelerators (Shader::initializeAccelerators + rayTrace / shadowTrace) ------------------ */
void *ref_trace_create(const MrtSceneDesc *desc, int accel, const float *camera_position) {
    auto h = std::make_unique<TraceHandle>();
    h->accel = accel;
    h->n_tri = desc->n_triangles;
    h->n_sph = desc->n_spheres;
    h->n_pln = desc->n_planes;
    h->n_lights = desc->n_lights;
    MrtCamera cam{};
    for (int k = 0; k < 3; ++k) cam.position[k] = camera_position[k];
    cam.look_at[0] = camera_position[0];
    cam.look_at[1] = camera_position[1];
    cam.look_at[2] = camera_position[2] + 1.0f;
    cam.up[1] = 1.0f;
    cam.fov_h_deg = 45.0f;
    cam.fov_v_deg = 45.0f;
    h->camera = make_camera(cam);
    h->shader = std::make_unique<IdShader>(make_scene(*desc, MRT_SAMPLER_RANDOM, 0.5f, 16, 16, 1),
                                           static_cast<Shader::Accelerator>(accel));
    h->shader->initializeAccelerators(h->camera.get());
    return h.release();
}

void ref_trace_destroy(void *handle) { delete static_cast<TraceHandle *>(handle); }

int ref_trace_closest(void *handle, const MrtRay *rays, uint32_t n, MrtHit *hits, int threads) {
    TraceHandle &h = *static_cast<TraceHandle *>(handle);
    parallel_for(n, threads, [&](uint32_t i) {
        const MrtRay &r = rays[i];
        const Ray ray{v3(r.direction), v3(r.origin), r.depth, exclude_pointer(h, r.exclude)};
        tl_record.hit = false;
        ::glm::vec3 rgb{};
        h.shader->rayTrace(&rgb, ray);
        if (tl_record.hit) {
            hits[i].t = tl_record.length;
            hits[i].id = identify(h, ray, tl_record);
        } else {
            hits[i].t = ::MobileRT::RayLengthMax;
            hits[i].id = MRT_HIT_NONE;
        }
    });
    return 0;
}

int ref_trace_any(void *handle, const MrtRay *rays, const float *dist, uint32_t n, uint8_t *occluded, int threads) {
    TraceHandle &h = *static_cast<TraceHandle *>(handle);
    parallel_for(n, threads, [&](uint32_t i) {
        const MrtRay &r = rays[i];
        const Ray ray{v3(r.direction), v3(r.origin), r.depth, exclude_pointer(h, r.exclude)};
        occluded[i] = h.shader->shadowTrace(ray, dist[i]) ? 1 : 0;
    });
    return 0;
}

/* ---- whole frames ----------------------------------------------------------------------------- */
// Renderer construction (accelerator build) and renderFrame, timed as c_wrapper.cpp:493-523 does.
int ref_render(const MrtSceneDesc *desc, const MrtCamera *camera, const MrtRenderOpts *o, int accel, int threads,
               uint32_t *bitmap, uint32_t stride, double *t_build, double *t_render) {
    Scene scene = make_scene(*desc, o->light_sampler, o->constant_value, o->width, o->height, o->spp);
    auto shader = make_shader(std::move(scene), *o, accel);
    const auto t0 = std::chrono::steady_clock::now();
    ::MobileRT::Renderer renderer{std::move(shader), make_camera(*camera),
                                  make_sampler(o->pixel_sampler, o->constant_value, o->width, o->height, o->spp),
                                  o->width, o->height, o->spp};
    if (t_build) *t_build = seconds_since(t0);
    const auto t1 = std::chrono::steady_clock::now();
    renderer.renderFrame(bitmap, threads, stride);
    if (t_render) *t_render = seconds_since(t1);
    return 0;
}

// The per-pixel body of Renderer::renderScene (Renderer.cpp:94-108) on the reference's own camera,
// sampler and shader objects, over every `pixel_step`-th pixel in scanline order starting at
// `pixel_first`, sample 0 only.  Used to time a bounded sample of a frame too large to render whole
// on the CPU; returns the number of camera rays traced.
uint64_t ref_render_subset(const MrtSceneDesc *desc, const MrtCamera *camera, const MrtRenderOpts *o, int accel,
                           int threads, uint32_t pixel_first, uint32_t pixel_step, uint32_t *bitmap,
                           double *t_build, double *t_render) {
    Scene scene = make_scene(*desc, o->light_sampler, o->constant_value, o->width, o->height, o->spp);
    auto shader = make_shader(std::move(scene), *o, accel);
    auto cam = make_camera(*camera);
    auto sampler = make_sampler(o->pixel_sampler, o->constant_value, o->width, o->height, o->spp);
    const auto t0 = std::chrono::steady_clock::now();
    shader->initializeAccelerators(cam.get());
    if (t_build) *t_build = seconds_since(t0);
    const uint32_t w = o->width, hgt = o->height;
    const uint64_t total = static_cast<uint64_t>(w) * hgt;
    const uint32_t count = pixel_first >= total ? 0u : static_cast<uint32_t>((total - pixel_first + pixel_step - 1) / pixel_step);
    const float inv_w = 1.0f / w, inv_h = 1.0f / hgt, pw = 0.5f / w, ph = 0.5f / hgt;
    const auto t1 = std::chrono::steady_clock::now();
    parallel_for(count, threads, [&](uint32_t k) {
        const uint64_t p = pixel_first + static_cast<uint64_t>(k) * pixel_step;
        const uint32_t x = static_cast<uint32_t>(p % w), y = static_cast<uint32_t>(p / w);
        const float u = x * inv_w, v = y * inv_h;
        const float r1 = sampler->getSample(), r2 = sampler->getSample();
        const Ray ray = cam->generateRay(u, v, (r1 - 0.5f) * 2.0f * pw, (r2 - 0.5f) * 2.0f * ph);
        ::glm::vec3 rgb{};
        shader->rayTrace(&rgb, ray);
        if (bitmap) bitmap[k] = ::MobileRT::incrementalAvg(rgb, bitmap[k], 1);
    });
    if (t_render) *t_render = seconds_since(t1);
    return count;
}

/* ---- OBJ scenes -------------------------------------------------------------------------------- */
// The reference's OBJLoader::process and OBJLoader::fillScene on a parse the caller stages (vertices
// with colours, normals, triangulated faces with their material ids, materials): the loader's own
// conversion code builds the Scene.  Outputs, per scene triangle 30 floats (A, AB, AC, normals A B C,
// colours A B C, material index as int bits), per material 13 (Le, Kd, Ks, Kt, ior), per area light 22
// (its triangle's A, AB, AC, then its material's 13).  counts: triangles, materials, lights.
int ref_obj_fill(const char *obj_path, const char *mtl_path, const float *vertices, const float *colors, uint32_t nv,
                 const float *normals, uint32_t nn, const int32_t *face_idx, const int32_t *face_mat, uint32_t n_faces,
                 const float *mats, uint32_t n_mat, float *out_tri, float *out_mat, float *out_light, uint32_t *counts) {
    ObjStage &st = obj_stage();
    st = ObjStage{};
    st.attrib.vertices.assign(vertices, vertices + 3ull * nv);
    st.attrib.colors.assign(colors, colors + 3ull * nv);
    if (nn) st.attrib.normals.assign(normals, normals + 3ull * nn);
    ::tinyobj::shape_t shape;
    shape.name = "staged";
    for (uint32_t f = 0; f < n_faces; ++f) {
        for (int k = 0; k < 3; ++k)
            shape.mesh.indices.push_back(::tinyobj::index_t{face_idx[6 * f + 2 * k], face_idx[6 * f + 2 * k + 1], -1});
        shape.mesh.num_face_vertices.push_back(3u);
        shape.mesh.material_ids.push_back(face_mat[f]);
    }
    st.shapes.push_back(std::move(shape));
    for (uint32_t m = 0; m < n_mat; ++m) {
        const float *x = mats + 14ull * m;
        ::tinyobj::material_t t{};
        for (int k = 0; k < 3; ++k) {
            t.diffuse[k] = x[k];
            t.specular[k] = x[3 + k];
            t.transmittance[k] = x[6 + k];
            t.emission[k] = x[9 + k];
        }
        t.ior = x[12];
        t.dissolve = x[13];
        st.materials.push_back(t);
    }
    st.staged = true;
    Scene scene{};
    {
        ::Components::OBJLoader loader{obj_path, mtl_path ? mtl_path : ""};
        if (loader.process() < 0 || !loader.isProcessed()) return 1;
        if (!loader.fillScene(&scene, [] { return std::make_unique<::Components::Constant>(0.5f); })) return 2;
    }
    st = ObjStage{};
    auto put3 = [](float *o, const ::glm::vec3 &v) { o[0] = v[0]; o[1] = v[1]; o[2] = v[2]; };
    auto put_mat = [&](float *o, const Material &m) {
        put3(o, m.Le_); put3(o + 3, m.Kd_); put3(o + 6, m.Ks_); put3(o + 9, m.Kt_); o[12] = m.refractiveIndice_;
    };
    auto put_tri = [&](float *o, const Triangle &t) { put3(o, t.pointA_); put3(o + 3, t.AB_); put3(o + 6, t.AC_); };
    for (size_t i = 0; i < scene.triangles_.size(); ++i) {
        const Triangle &t = scene.triangles_[i];
        float *o = out_tri + 30 * i;
        put_tri(o, t);
        put3(o + 9, t.normalA_); put3(o + 12, t.normalB_); put3(o + 15, t.normalC_);
        put3(o + 18, t.colorA_); put3(o + 21, t.colorB_); put3(o + 24, t.colorC_);
        std::memcpy(o + 27, &t.materialId_, 4);
        o[28] = o[29] = 0.0f;
    }
    for (size_t i = 0; i < scene.materials_.size(); ++i) put_mat(out_mat + 13 * i, scene.materials_[i]);
    for (size_t i = 0; i < scene.lights_.size(); ++i) {
        const auto *al = dynamic_cast<const ::Components::AreaLight *>(scene.lights_[i].get());
        if (!al) return 3;
        put_tri(out_light + 22 * i, al->*get(AreaLightTriangle{}));
        put_mat(out_light + 22 * i + 9, al->radiance_);
    }
    counts[0] = static_cast<uint32_t>(scene.triangles_.size());
    counts[1] = static_cast<uint32_t>(scene.materials_.size());
    counts[2] = static_cast<uint32_t>(scene.lights_.size());
    return 0;
}

}  // extern "C"
