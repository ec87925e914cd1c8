// A client that loads its scene the way the reference's Linux driver does for OBJ files
// (c_wrapper.cpp: OBJLoader::process, fillScene with a light-sampler factory, then Shader, Camera,
// Renderer, renderFrame), compiled against the drop-in headers and libmrt_dropin.so.
//
//   dropin_obj <scene.obj> <scene.mtl> <shader 1|3|4> <orthographic 0|1> <width> <height> <out.bin>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "Components/Cameras/Orthographic.hpp"
#include "Components/Cameras/Perspective.hpp"
#include "Components/ObjectLoaders/OBJLoader.hpp"
#include "Components/Samplers/Constant.hpp"
#include "Components/Samplers/MersenneTwister.hpp"
#include "Components/Shaders/DepthMap.hpp"
#include "Components/Shaders/DiffuseMaterial.hpp"
#include "Components/Shaders/Whitted.hpp"
#include "MobileRT/Renderer.hpp"
#include "MobileRT/Scene.hpp"

int main(int argc, char **argv) {
    if (argc != 8) { std::fprintf(stderr, "usage: dropin_obj obj mtl shader ortho width height out\n"); return 2; }
    const int shaderKind = std::atoi(argv[3]), ortho = std::atoi(argv[4]);
    const std::uint32_t width = (std::uint32_t)std::atoi(argv[5]), height = (std::uint32_t)std::atoi(argv[6]);
    ::Components::OBJLoader loader{argv[1], argv[2]};
    if (loader.process() < 0) { std::fprintf(stderr, "%s\n", loader.lastError().c_str()); return 3; }
    ::MobileRT::Scene scene{};
    if (!loader.fillScene(&scene, []() { return std::make_unique<::Components::MersenneTwister>(); })) return 4;
    const auto accel = ::MobileRT::Shader::Accelerator::BVH;
    std::unique_ptr<::MobileRT::Shader> shader;
    if (shaderKind == 3) shader = std::make_unique<::Components::DepthMap>(std::move(scene), ::glm::vec3{1.5f, 1.0f, 2.0f}, accel);
    else if (shaderKind == 4) shader = std::make_unique<::Components::DiffuseMaterial>(std::move(scene), accel);
    else shader = std::make_unique<::Components::Whitted>(std::move(scene), 1, accel);
    std::unique_ptr<::MobileRT::Camera> camera;
    if (ortho) camera = std::make_unique<::Components::Orthographic>(::glm::vec3{0.0f, 0.1f, -2.6f}, ::glm::vec3{0.0f, 0.0f, 1.0f},
                                                                      ::glm::vec3{0.0f, 1.0f, 0.0f}, 2.4f, 2.0f);
    else camera = std::make_unique<::Components::Perspective>(::glm::vec3{0.0f, 0.1f, -2.6f}, ::glm::vec3{0.0f, 0.0f, 1.0f},
                                                               ::glm::vec3{0.0f, 1.0f, 0.0f}, 55.0f, 55.0f);
    ::MobileRT::Renderer renderer{std::move(shader), std::move(camera), std::make_unique<::Components::Constant>(0.5f),
                                  width, height, 1};
    std::vector<std::uint32_t> bitmap(width * height, 0u);
    renderer.renderFrame(bitmap.data(), 8, width * 4);
    if (!renderer.lastError().empty()) { std::fprintf(stderr, "%s\n", renderer.lastError().c_str()); return 5; }
    FILE *out = std::fopen(argv[7], "wb");
    if (!out) return 6;
    std::fwrite(bitmap.data(), 4, bitmap.size(), out);
    std::fclose(out);
    return 0;
}
