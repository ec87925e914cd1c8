// A client written against the MobileRT API the way the reference's Linux driver is
// (app/System_dependent/Linux/c_wrapper.cpp: build Scene, Camera, samplers, Shader, Renderer, then
// renderFrame), compiled against the drop-in headers and libmrt_dropin.so.
//
//   dropin_render <scene.bin> <out.bin>
// scene.bin (little endian, written by tests/test_gpu_dropin.py): triangles, spheres, planes,
// materials, lights, camera and render options; out.bin: the ARGB8888 bitmap, row-major.
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "Components/Cameras/Perspective.hpp"
#include "Components/Lights/AreaLight.hpp"
#include "Components/Lights/PointLight.hpp"
#include "Components/Samplers/Constant.hpp"
#include "Components/Samplers/HaltonSeq.hpp"
#include "Components/Samplers/MersenneTwister.hpp"
#include "Components/Samplers/Stratified.hpp"
#include "Components/Shaders/NoShadows.hpp"
#include "Components/Shaders/PathTracer.hpp"
#include "Components/Shaders/Whitted.hpp"
#include "MobileRT/Renderer.hpp"
#include "MobileRT/Scene.hpp"

namespace {
FILE *in;
template <typename T> T rd() {
    T v{};
    if (std::fread(&v, sizeof(T), 1, in) != 1) { std::fprintf(stderr, "short read\n"); std::exit(2); }
    return v;
}
::glm::vec3 v3() {
    const float x = rd<float>(), y = rd<float>(), z = rd<float>();
    return ::glm::vec3{x, y, z};
}
std::unique_ptr<MobileRT::Sampler> sampler(int kind, float value) {
    switch (kind) {
        case 0: return std::make_unique<Components::Constant>(value);
        case 1: return std::make_unique<Components::Stratified>();
        case 2: return std::make_unique<Components::HaltonSeq>();
        default: return std::make_unique<Components::MersenneTwister>();
    }
}
MobileRT::Material material() {
    const ::glm::vec3 le = v3(), kd = v3(), ks = v3(), kt = v3();
    const float ior = rd<float>();
    return MobileRT::Material{kd, ks, kt, ior, le};
}
}  // namespace

int main(int argc, char **argv) {
    if (argc != 3 && argc != 4) { std::fprintf(stderr, "usage: %s scene.bin out.bin [preview.bin]\n", argv[0]); return 1; }
    in = std::fopen(argv[1], "rb");
    if (!in) return 1;
    MobileRT::Scene scene{};
    const uint32_t nt = rd<uint32_t>(), has_n = rd<uint32_t>(), has_c = rd<uint32_t>();
    for (uint32_t i = 0; i < nt; ++i) {
        const ::glm::vec3 a = v3(), b = v3(), c = v3();
        ::glm::vec3 n[3], col[3];
        if (has_n) for (auto &x : n) x = v3();
        if (has_c) for (auto &x : col) x = v3();
        const int32_t mat = rd<int32_t>();
        if (has_n) scene.triangles_.emplace_back(MobileRT::Triangle{a, b, c, mat, n[0], n[1], n[2], col[0], col[1], col[2]});
        else if (has_c) scene.triangles_.emplace_back(MobileRT::Triangle{a, b, c, mat, col[0], col[1], col[2]});
        else scene.triangles_.emplace_back(MobileRT::Triangle{a, b, c, mat});
    }
    const uint32_t ns = rd<uint32_t>();
    for (uint32_t i = 0; i < ns; ++i) {
        const ::glm::vec3 c = v3();
        const float r = rd<float>();
        scene.spheres_.emplace_back(MobileRT::Sphere{c, r, rd<int32_t>()});
    }
    const uint32_t np = rd<uint32_t>();
    for (uint32_t i = 0; i < np; ++i) {
        const ::glm::vec3 p = v3(), n = v3();
        scene.planes_.emplace_back(MobileRT::Plane{p, n, rd<int32_t>()});
    }
    const uint32_t nm = rd<uint32_t>();
    for (uint32_t i = 0; i < nm; ++i) scene.materials_.emplace_back(material());
    const uint32_t nl = rd<uint32_t>();
    std::vector<int> light_kinds;
    for (uint32_t i = 0; i < nl; ++i) {
        const int32_t kind = rd<int32_t>();
        const ::glm::vec3 p0 = v3(), p1 = v3(), p2 = v3();
        const MobileRT::Material m = material();
        light_kinds.push_back(kind);
        if (kind == 1) scene.lights_.emplace_back(std::make_unique<Components::AreaLight>(m, nullptr, p0, p1, p2));
        else scene.lights_.emplace_back(std::make_unique<Components::PointLight>(m, p0));
    }
    const ::glm::vec3 pos = v3(), look = v3(), up = v3();
    const float hfov = rd<float>(), vfov = rd<float>();
    const int32_t shader_kind = rd<int32_t>(), accel = rd<int32_t>(), bvh_mode = rd<int32_t>();
    const uint32_t w = rd<uint32_t>(), h = rd<uint32_t>(), spp = rd<uint32_t>(), spl = rd<uint32_t>();
    const int32_t pix_kind = rd<int32_t>();
    const float cval = rd<float>();
    const int32_t light_kind = rd<int32_t>(), rr_kind = rd<int32_t>();
    std::fclose(in);
    for (auto &l : scene.lights_)   // area lights get their sampler (AreaLight.cpp:13-19)
        if (l->isArea()) static_cast<Components::AreaLight *>(l.get())->samplerPointLight_ = sampler(light_kind, cval);

    std::unique_ptr<MobileRT::Shader> shader;
    const auto a = static_cast<MobileRT::Shader::Accelerator>(accel);
    if (shader_kind == 1) shader = std::make_unique<Components::Whitted>(std::move(scene), spl, a);
    else if (shader_kind == 2) shader = std::make_unique<Components::PathTracer>(std::move(scene), sampler(rr_kind, cval), spl, a);
    else shader = std::make_unique<Components::NoShadows>(std::move(scene), spl, a);
    shader->setBvhMode(bvh_mode);
    auto camera = std::make_unique<Components::Perspective>(pos, look, up, hfov, vfov);
    MobileRT::Renderer renderer{std::move(shader), std::move(camera), sampler(pix_kind, cval), w, h, spp};
    std::vector<uint32_t> bitmap(static_cast<size_t>(w) * h, 0u);
    renderer.renderFrame(bitmap.data(), 8, w * sizeof(uint32_t));
    if (!renderer.lastError().empty()) { std::fprintf(stderr, "%s\n", renderer.lastError().c_str()); return 3; }
    FILE *out = std::fopen(argv[2], "wb");
    std::fwrite(bitmap.data(), sizeof(uint32_t), bitmap.size(), out);
    std::fclose(out);
    if (argc == 4) {   // the front end's raster preview of the same renderer
        std::vector<uint32_t> preview(static_cast<size_t>(w) * h, 0u);
        renderer.rasterPreview(preview.data(), w * sizeof(uint32_t));
        if (!renderer.lastError().empty()) { std::fprintf(stderr, "%s\n", renderer.lastError().c_str()); return 4; }
        FILE *pv = std::fopen(argv[3], "wb");
        std::fwrite(preview.data(), sizeof(uint32_t), preview.size(), pv);
        std::fclose(pv);
    }
    std::printf("rendered %ux%u, samples %u\n", w, h, renderer.getSample());
    return 0;
}
