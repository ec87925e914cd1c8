// dropin.cpp - the MobileRT render API of b200_api.hpp over the C ABI of include/mrt_cuda.h.
// Built with -ffp-contract=off (python -m mobileraytracer_b200.build_dropin) so the normals it
// computes for triangles without given normals round like the reference's constructors.
#include "MobileRT/b200_api.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "../../../include/mrt_cuda.h"

namespace MobileRT {

struct DeviceScene {
    MrtScene *scene = nullptr;
};

namespace {

// one context per process on the device named by MRT_DEVICE (default 0)
MrtContext *context() {
    static std::once_flag once;
    static MrtContext *ctx = nullptr;
    std::call_once(once, [] {
        const char *e = std::getenv("MRT_DEVICE");
        if (mrt_context_create(e ? std::atoi(e) : 0, &ctx) != MRT_OK) ctx = nullptr;
    });
    return ctx;
}

MrtCamera to_mrt(const Camera &camera) {
    MrtCamera c{};
    c.kind = camera.kind();
    for (int k = 0; k < 3; ++k) { c.position[k] = camera.position_.v[k]; c.look_at[k] = camera.lookAt_.v[k]; c.up[k] = camera.up_.v[k]; }
    c.fov_h_deg = camera.hFovDegrees();
    c.fov_v_deg = camera.vFovDegrees();
    return c;
}

std::string context_error(MrtContext *ctx, int st, const char *what) {
    return std::string(what) + ": status " + std::to_string(st) + ": " + (ctx ? mrt_context_error(ctx) : "no CUDA context");
}

void put(float *dst, const detail::F3 &v) { dst[0] = v.v[0]; dst[1] = v.v[1]; dst[2] = v.v[2]; }
void put(float *dst, const ::glm::vec3 &v) { dst[0] = v[0]; dst[1] = v[1]; dst[2] = v[2]; }

void material_of(const Material &m, MrtMaterial &o) {
    put(o.le, m.Le_); put(o.kd, m.Kd_); put(o.ks, m.Ks_); put(o.kt, m.Kt_);
    o.ior = m.refractiveIndice_;
}

int sampler_kind(const Sampler *s) { return s ? (int)s->kind() : MRT_SAMPLER_RANDOM; }

}  // namespace

float Sampler::getSample(std::uint32_t /*sample*/) noexcept {
    switch (kind_) {
        case CONSTANT: return value_;
        default: {   // a 32-bit avalanche hash of a counter (host-side draws are not used by the GPU path)
            std::uint32_t x = ++counter_ * 0x9e3779b9u;
            x ^= x >> 16; x *= 0x21f0aaadu; x ^= x >> 15; x *= 0x735a2d97u; x ^= x >> 15;
            return (float)(x >> 8) * (1.0f / 16777216.0f);
        }
    }
}

Shader::Shader(Scene &&scene, std::uint32_t samplesLight, Accelerator accelerator) noexcept
    : scene_{std::move(scene)}, samplesLight_{samplesLight}, accelerator_{accelerator} {}

Shader::~Shader() noexcept {
    if (device_) {
        mrt_scene_destroy(device_->scene);
        delete device_;
    }
}

void Shader::initializeAccelerators(Camera *camera) noexcept {
    MrtContext *ctx = context();
    if (!ctx) { error_ = "no CUDA device"; std::fprintf(stderr, "MobileRT: %s\n", error_.c_str()); return; }
    const std::size_t nt = scene_.triangles_.size();
    std::vector<float> abc(9 * nt), nrm(9 * nt), col(9 * nt);
    std::vector<std::int32_t> tmat(nt);
    for (std::size_t i = 0; i < nt; ++i) {
        const Triangle &t = scene_.triangles_[i];
        put(&abc[9 * i], t.pointA_);
        put(&abc[9 * i + 3], t.b_);
        put(&abc[9 * i + 6], t.c_);
        if (t.givenNormals_) {
            put(&nrm[9 * i], t.normalA_); put(&nrm[9 * i + 3], t.normalB_); put(&nrm[9 * i + 6], t.normalC_);
        } else {   // normalize(cross(AC, AB)), Triangle.cpp:10-21, glm order v * (1 / sqrt(dot(v, v)))
            const float A[3] = {abc[9 * i], abc[9 * i + 1], abc[9 * i + 2]};
            const float ac[3] = {abc[9 * i + 6] - A[0], abc[9 * i + 7] - A[1], abc[9 * i + 8] - A[2]};
            const float ab[3] = {abc[9 * i + 3] - A[0], abc[9 * i + 4] - A[1], abc[9 * i + 5] - A[2]};
            const float c[3] = {ac[1] * ab[2] - ab[1] * ac[2], ac[2] * ab[0] - ab[2] * ac[0], ac[0] * ab[1] - ab[0] * ac[1]};
            const float px = c[0] * c[0], py = c[1] * c[1], pz = c[2] * c[2];
            const float inv = 1.0f / std::sqrt((px + py) + pz);
            for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) nrm[9 * i + 3 * k + j] = c[j] * inv;
        }
        put(&col[9 * i], t.colorA_); put(&col[9 * i + 3], t.colorB_); put(&col[9 * i + 6], t.colorC_);
        tmat[i] = t.materialId_;
    }
    std::vector<float> sph(4 * scene_.spheres_.size()), pln(6 * scene_.planes_.size());
    std::vector<std::int32_t> smat(scene_.spheres_.size()), pmat(scene_.planes_.size());
    for (std::size_t i = 0; i < scene_.spheres_.size(); ++i) {
        put(&sph[4 * i], scene_.spheres_[i].center_);
        sph[4 * i + 3] = scene_.spheres_[i].radius_;
        smat[i] = scene_.spheres_[i].materialId_;
    }
    for (std::size_t i = 0; i < scene_.planes_.size(); ++i) {
        put(&pln[6 * i], scene_.planes_[i].point_);
        put(&pln[6 * i + 3], scene_.planes_[i].normal_);
        pmat[i] = scene_.planes_[i].materialId_;
    }
    std::vector<MrtMaterial> mats(scene_.materials_.size());
    for (std::size_t i = 0; i < mats.size(); ++i) material_of(scene_.materials_[i], mats[i]);
    std::vector<MrtLightDesc> lights(scene_.lights_.size());
    for (std::size_t i = 0; i < lights.size(); ++i) {
        const Light *l = scene_.lights_[i].get();
        MrtLightDesc &o = lights[i];
        material_of(l->radiance_, o.radiance);
        if (l->isArea()) {
            const auto *a = static_cast<const Components::AreaLight *>(l);
            o.kind = MRT_LIGHT_AREA;
            put(o.p0, a->a_); put(o.p1, a->b_); put(o.p2, a->c_);
        } else {
            const auto *p = static_cast<const Components::PointLight *>(l);
            o.kind = MRT_LIGHT_POINT;
            put(o.p0, p->position_);
            put(o.p1, p->position_); put(o.p2, p->position_);
        }
    }
    MrtSceneDesc d{};
    d.n_triangles = (std::uint32_t)nt;
    d.tri_abc = abc.data(); d.tri_normals = nrm.data(); d.tri_colors = col.data(); d.tri_material = tmat.data();
    d.n_spheres = (std::uint32_t)smat.size(); d.sphere_center_radius = sph.data(); d.sphere_material = smat.data();
    d.n_planes = (std::uint32_t)pmat.size(); d.plane_point_normal = pln.data(); d.plane_material = pmat.data();
    d.n_materials = (std::uint32_t)mats.size(); d.materials = mats.data();
    d.n_lights = (std::uint32_t)lights.size(); d.lights = lights.data();
    if (device_) { mrt_scene_destroy(device_->scene); delete device_; device_ = nullptr; }
    MrtScene *s = nullptr;
    int st = mrt_scene_create(ctx, &d, &s);
    if (st != MRT_OK) { error_ = context_error(ctx, st, "mrt_scene_create"); std::fprintf(stderr, "MobileRT: %s\n", error_.c_str()); return; }
    MrtAccelOpts o{};
    o.accelerator = (std::int32_t)accelerator_;
    o.bvh_mode = bvhMode_;
    o.grid_size = gridSize_;
    o.grid_index = gridIndex_;
    MrtCamera cam{};
    if (camera) {
        o.camera_position[0] = camera->position_.v[0]; o.camera_position[1] = camera->position_.v[1]; o.camera_position[2] = camera->position_.v[2];
        cam = to_mrt(*camera);
        o.camera = &cam;   // grid bounds take the camera's getAABB (Shader.cpp:56-62)
    }
    st = mrt_scene_build(s, &o);
    if (st != MRT_OK) {
        error_ = context_error(ctx, st, "mrt_scene_build");
        std::fprintf(stderr, "MobileRT: %s\n", error_.c_str());
        mrt_scene_destroy(s);
        return;
    }
    device_ = new DeviceScene{s};
}

Renderer::Renderer(std::unique_ptr<Shader> shader, std::unique_ptr<Camera> camera, std::unique_ptr<Sampler> samplerPixel,
                   std::uint32_t width, std::uint32_t height, std::uint32_t samplesPixel) noexcept
    : camera_{std::move(camera)}, shader_{std::move(shader)}, samplerPixel_{std::move(samplerPixel)}, width_{width},
      height_{height}, samplesPixel_{samplesPixel} {
    shader_->initializeAccelerators(camera_.get());   // Renderer.cpp:28
}

void Renderer::renderFrame(std::uint32_t *bitmap, std::int32_t /*numThreads*/, std::uint32_t stride) noexcept {
    if (!shader_ || !shader_->device_) {
        error_ = shader_ ? shader_->error_ : "no shader";
        std::fprintf(stderr, "MobileRT: renderFrame without an uploaded scene: %s\n", error_.c_str());
        return;
    }
    MrtRenderOpts o{};
    o.shader = shader_->shaderKind();
    o.width = width_;
    o.height = height_;
    o.spp = samplesPixel_;
    o.spl = shader_->samplesLight();
    o.pixel_sampler = sampler_kind(samplerPixel_.get());
    o.constant_value = samplerPixel_ ? samplerPixel_->value() : 0.5f;
    o.light_sampler = MRT_SAMPLER_RANDOM;
    for (const auto &l : shader_->scene_.lights_)
        if (l->isArea()) { o.light_sampler = sampler_kind(static_cast<const Components::AreaLight *>(l.get())->samplerPointLight_.get()); break; }
    o.rr_sampler = sampler_kind(shader_->russianRoulette());
    o.depth_min = depthMin_;
    o.depth_max = depthMax_;
    o.seed = seed_;
    const detail::F3 dp = shader_->depthPoint();
    for (int k = 0; k < 3; ++k) o.depth_point[k] = dp.v[k];
    const MrtCamera c = to_mrt(*camera_);
    const int st = mrt_render(shader_->device_->scene, &c, &o, bitmap, stride, nullptr, MRT_MEM_HOST, nullptr);
    if (st != MRT_OK && st != MRT_ERR_CANCELLED) {
        error_ = context_error(context(), st, "mrt_render");
        std::fprintf(stderr, "MobileRT: %s\n", error_.c_str());
    }
}

void Renderer::stopRender() noexcept {
    if (shader_ && shader_->device_) mrt_render_stop(shader_->device_->scene);
}

void Renderer::rasterPreview(std::uint32_t *bitmap, std::uint32_t stride) noexcept {
    if (!shader_ || !shader_->device_) {
        error_ = shader_ ? shader_->error_ : "no shader";
        std::fprintf(stderr, "MobileRT: rasterPreview without an uploaded scene: %s\n", error_.c_str());
        return;
    }
    const MrtCamera c = to_mrt(*camera_);
    const int st = mrt_raster_preview(shader_->device_->scene, &c, width_, height_, bitmap, stride, MRT_MEM_HOST, nullptr);
    if (st != MRT_OK) {
        error_ = context_error(context(), st, "mrt_raster_preview");
        std::fprintf(stderr, "MobileRT: %s\n", error_.c_str());
    }
}

std::uint32_t Renderer::getSample() const noexcept {
    return (shader_ && shader_->device_) ? mrt_render_progress(shader_->device_->scene) : 0u;
}

}  // namespace MobileRT

namespace Components {

namespace {
struct ObjData {
    MrtObjScene *scene{nullptr};
    MrtSceneDesc desc{};
    ~ObjData() { if (scene) mrt_obj_free(scene); }
};
}  // namespace

OBJLoader::OBJLoader(std::string obj, std::string materials) noexcept
    : objFilePath_{std::move(obj)}, mtlFilePath_{std::move(materials)} {}

OBJLoader::~OBJLoader() noexcept { delete static_cast<ObjData *>(data_); }

std::int32_t OBJLoader::process() noexcept {
    delete static_cast<ObjData *>(data_);
    ObjData *o = new ObjData();
    data_ = o;
    char err[512] = {0};
    const int st = mrt_obj_load(objFilePath_.c_str(), mtlFilePath_.empty() ? nullptr : mtlFilePath_.c_str(), &o->scene,
                                &o->desc, err, sizeof(err));
    isProcessed_ = st == MRT_OK;
    error_ = isProcessed_ ? std::string{} : std::string{err};
    numberTriangles_ = isProcessed_ ? (std::int32_t)(o->desc.n_triangles + o->desc.n_lights) : -1;
    return numberTriangles_;
}

bool OBJLoader::fillScene(::MobileRT::Scene *scene, std::function<std::unique_ptr<::MobileRT::Sampler>()> lambda) noexcept {
    if (!isProcessed_ || !data_ || !scene) return false;
    const MrtSceneDesc &d = static_cast<ObjData *>(data_)->desc;
    auto v = [](const float *p) { return ::glm::vec3{p[0], p[1], p[2]}; };
    auto mat = [&](const MrtMaterial &m) {
        return ::MobileRT::Material{v(m.kd), v(m.ks), v(m.kt), m.ior, v(m.le)};
    };
    const std::size_t m0 = scene->materials_.size();
    for (std::uint32_t i = 0; i < d.n_materials; ++i) scene->materials_.emplace_back(mat(d.materials[i]));
    scene->triangles_.reserve(scene->triangles_.size() + d.n_triangles);
    for (std::uint32_t i = 0; i < d.n_triangles; ++i) {
        const float *p = d.tri_abc + 9 * (std::size_t)i, *n = d.tri_normals + 9 * (std::size_t)i,
                    *c = d.tri_colors + 9 * (std::size_t)i;
        const std::int32_t m = d.tri_material[i] < 0 ? -1 : d.tri_material[i] + (std::int32_t)m0;
        scene->triangles_.emplace_back(v(p), v(p + 3), v(p + 6), m, v(n), v(n + 3), v(n + 6), v(c), v(c + 3), v(c + 6));
    }
    for (std::uint32_t i = 0; i < d.n_lights; ++i) {
        const MrtLightDesc &l = d.lights[i];
        scene->lights_.emplace_back(std::make_unique<AreaLight>(mat(l.radiance), lambda(), v(l.p0), v(l.p1), v(l.p2)));
    }
    return true;
}

}  // namespace Components
