// b200_api.hpp - the MobileRT render API (Scene / Shader / Sampler / Camera / Renderer) with the
// work done by the B200 path behind include/mrt_cuda.h.
//
// Class names, header paths, constructors and the members callers use are those of the reference
// (app/MobileRT/*.hpp, app/Components/*/*.hpp), so code written against the reference compiles
// unchanged against these headers and libmrt_dropin.so:
//
//     auto shader = std::make_unique<Components::Whitted>(std::move(scene), samplesLight, Shader::BVH);
//     MobileRT::Renderer renderer {std::move(shader), std::move(camera), std::move(sampler), w, h, spp};
//     renderer.renderFrame(bitmap, numThreads, w * sizeof(uint32_t));
//
// The scene is uploaded and the accelerator built when the Renderer is constructed
// (Shader::initializeAccelerators, Shader.cpp:31-122); renderFrame runs on the GPU and writes the
// same ARGB8888 running mean into the caller's bitmap.  Every call stays noexcept as in the
// reference: a failure is logged, leaves the bitmap untouched and is kept in lastError().
//
// glm::vec3 appears only in inline code of these headers (the caller's GLM); the library itself
// receives plain floats.
#ifndef MRT_B200_API_HPP
#define MRT_B200_API_HPP

#include <glm/glm.hpp>

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

namespace MobileRT {

const float RayLengthMax{1.0e+30f};   // Utils.hpp:33-37
const std::int32_t RayDepthMin{4};
const std::int32_t RayDepthMax{8};
const std::int32_t NumberOfBlocks{256};
const float Epsilon{1.0e-06f};

namespace detail {
struct F3 {
    float v[3];
};
inline F3 f3(const ::glm::vec3 &a) { return F3{{a[0], a[1], a[2]}}; }
}  // namespace detail

// Material.hpp:13-17
class Material final {
public:
    ::glm::vec3 Le_{};
    ::glm::vec3 Kd_{};
    ::glm::vec3 Ks_{};
    ::glm::vec3 Kt_{};
    float refractiveIndice_{};

    explicit Material() noexcept = default;
    explicit Material(const ::glm::vec3 &Kd, const ::glm::vec3 &Ks = ::glm::vec3{}, const ::glm::vec3 &Kt = ::glm::vec3{},
                      float refractiveIndice = 1.0f, const ::glm::vec3 &Le = ::glm::vec3{}) noexcept
        : Le_{Le}, Kd_{Kd}, Ks_{Ks}, Kt_{Kt}, refractiveIndice_{refractiveIndice} {}
};

// Triangle.hpp:14-66: the corner points are kept as given; AB_/AC_ are the reference's stored
// edges (B - A, C - A) and normals left unspecified are computed by the library exactly as the
// reference's constructors do (normalize(cross(AC, AB))).
class Triangle final {
public:
    ::glm::vec3 AC_{};
    ::glm::vec3 AB_{};
    ::glm::vec3 pointA_{};
    ::glm::vec3 normalA_{}, normalB_{}, normalC_{};
    ::glm::vec3 colorA_{}, colorB_{}, colorC_{};
    std::int32_t materialId_{};
    bool givenNormals_{false};
    detail::F3 b_{}, c_{};

    explicit Triangle(const ::glm::vec3 &a, const ::glm::vec3 &b, const ::glm::vec3 &c, std::int32_t materialId) noexcept
        : AC_{c - a}, AB_{b - a}, pointA_{a}, materialId_{materialId}, b_{detail::f3(b)}, c_{detail::f3(c)} {}
    explicit Triangle(const ::glm::vec3 &a, const ::glm::vec3 &b, const ::glm::vec3 &c, std::int32_t materialId,
                      const ::glm::vec3 &nA, const ::glm::vec3 &nB, const ::glm::vec3 &nC, const ::glm::vec3 &cA,
                      const ::glm::vec3 &cB, const ::glm::vec3 &cC) noexcept
        : AC_{c - a}, AB_{b - a}, pointA_{a}, normalA_{nA}, normalB_{nB}, normalC_{nC}, colorA_{cA}, colorB_{cB},
          colorC_{cC}, materialId_{materialId}, givenNormals_{true}, b_{detail::f3(b)}, c_{detail::f3(c)} {}
    explicit Triangle(const ::glm::vec3 &a, const ::glm::vec3 &b, const ::glm::vec3 &c, std::int32_t materialId,
                      const ::glm::vec3 &cA, const ::glm::vec3 &cB, const ::glm::vec3 &cC) noexcept
        : AC_{c - a}, AB_{b - a}, pointA_{a}, colorA_{cA}, colorB_{cB}, colorC_{cC}, materialId_{materialId},
          b_{detail::f3(b)}, c_{detail::f3(c)} {}
};

// Sphere.hpp:14-46
class Sphere final {
public:
    detail::F3 center_{};
    float radius_{};
    std::int32_t materialId_{};
    explicit Sphere(const ::glm::vec3 &center, float radius, std::int32_t materialId) noexcept
        : center_{detail::f3(center)}, radius_{radius}, materialId_{materialId} {}
};

// Plane.hpp:186-224 (the normal is normalised by the library, as Plane.cpp:11-15 does)
class Plane final {
public:
    detail::F3 point_{}, normal_{};
    std::int32_t materialId_{};
    explicit Plane(const ::glm::vec3 &point, const ::glm::vec3 &normal, std::int32_t materialId) noexcept
        : point_{detail::f3(point)}, normal_{detail::f3(normal)}, materialId_{materialId} {}
};

// Sampler.hpp:15-45.  Draws on the GPU are pure functions of (seed, pixel, sample, path node,
// dimension); getSample() on the host is provided for API completeness only.
class Sampler {
public:
    enum Kind { CONSTANT = 0, STRATIFIED = 1, HALTON = 2, RANDOM = 3 };
    explicit Sampler(Kind kind, float value = 0.5f) noexcept : kind_{kind}, value_{value} {}
    Sampler(const Sampler &) = delete;
    Sampler &operator=(const Sampler &) = delete;
    virtual ~Sampler() noexcept = default;
    void resetSampling() noexcept { counter_ = 0; }
    void stopSampling() noexcept {}
    virtual float getSample(std::uint32_t sample) noexcept;
    float getSample() noexcept { return getSample(0); }
    Kind kind() const noexcept { return kind_; }
    float value() const noexcept { return value_; }

private:
    Kind kind_;
    float value_;
    std::uint32_t counter_{0};
};

// Light.hpp:12-38
class Light {
public:
    const Material radiance_{};
    explicit Light(const Material &radiance) noexcept : radiance_{radiance} {}
    Light(const Light &) = delete;
    Light &operator=(const Light &) = delete;
    virtual ~Light() noexcept = default;
    virtual bool isArea() const noexcept = 0;
    virtual void resetSampling() noexcept {}
};

// Scene.hpp:20-55
class Scene final {
public:
    std::vector<Triangle> triangles_{};
    std::vector<Sphere> spheres_{};
    std::vector<Plane> planes_{};
    std::vector<Material> materials_{};
    std::vector<std::unique_ptr<Light>> lights_{};
    explicit Scene() = default;
    Scene(const Scene &) = delete;
    Scene(Scene &&) noexcept = default;
    Scene &operator=(Scene &&) noexcept = default;
    ~Scene() noexcept = default;
};

// Camera.hpp:12-57
class Camera {
public:
    detail::F3 position_{}, lookAt_{}, up_{};
    explicit Camera(const ::glm::vec3 &position, const ::glm::vec3 &lookAt, const ::glm::vec3 &up) noexcept
        : position_{detail::f3(position)}, lookAt_{detail::f3(lookAt)}, up_{detail::f3(up)} {}
    Camera(const Camera &) = delete;
    virtual ~Camera() noexcept = default;
    virtual int kind() const noexcept = 0;
    virtual float hFovDegrees() const noexcept = 0;
    virtual float vFovDegrees() const noexcept = 0;
    void resetSampling() noexcept {}
};

struct DeviceScene;   // the library's handle for an uploaded scene

// Shader.hpp:17-80
class Shader {
public:
    enum Accelerator { NAIVE = 0, REGULAR_GRID, BVH };
    Scene scene_{};

    explicit Shader(Scene &&scene, std::uint32_t samplesLight, Accelerator accelerator) noexcept;
    Shader(const Shader &) = delete;
    Shader &operator=(const Shader &) = delete;
    virtual ~Shader() noexcept;

    // Shader::initializeAccelerators (Shader.cpp:31-122): uploads the scene and builds the
    // accelerator on the GPU.  Called by the Renderer constructor.
    void initializeAccelerators(Camera *camera) noexcept;
    virtual void resetSampling() noexcept {}

    // which shade() the GPU runs (c_wrapper.cpp:444-486 codes: 0 NoShadows, 1 Whitted, 2 PathTracer,
    // 3 DepthMap, 4 DiffuseMaterial)
    virtual int shaderKind() const noexcept = 0;
    virtual const Sampler *russianRoulette() const noexcept { return nullptr; }
    virtual detail::F3 depthPoint() const noexcept { return detail::F3{}; }
    std::uint32_t samplesLight() const noexcept { return samplesLight_; }
    Accelerator accelerator() const noexcept { return accelerator_; }

    // extensions (not in the reference): BVH flavour (0 device-built fast tree, 1 reference tree),
    // RegularGrid size override (0 = the reference's rule) and cell addressing.
    void setBvhMode(int mode) noexcept { bvhMode_ = mode; }
    void setGridOptions(int gridSize, int gridIndex) noexcept { gridSize_ = gridSize; gridIndex_ = gridIndex; }
    DeviceScene *device() const noexcept { return device_; }
    const std::string &lastError() const noexcept { return error_; }

protected:
    std::uint32_t samplesLight_{};
    Accelerator accelerator_{};
    int bvhMode_{0};
    int gridSize_{0};
    int gridIndex_{0};
    DeviceScene *device_{nullptr};
    std::string error_{};
    friend class Renderer;
};

// Renderer.hpp:16-59
class Renderer final {
public:
    std::unique_ptr<Camera> camera_{};
    std::unique_ptr<Shader> shader_{};

    explicit Renderer(std::unique_ptr<Shader> shader, std::unique_ptr<Camera> camera,
                      std::unique_ptr<Sampler> samplerPixel, std::uint32_t width, std::uint32_t height,
                      std::uint32_t samplesPixel) noexcept;
    Renderer(const Renderer &) = delete;
    Renderer &operator=(const Renderer &) = delete;
    ~Renderer() noexcept = default;

    // Renderer::renderFrame (Renderer.cpp:31-59).  numThreads is accepted and ignored (the GPU
    // does the work); stride is the row pitch in bytes.
    void renderFrame(std::uint32_t *bitmap, std::int32_t numThreads, std::uint32_t stride) noexcept;
    void stopRender() noexcept;             // Renderer.cpp:61-65, callable from another thread
    std::uint32_t getSample() const noexcept;   // Renderer.cpp:118-120
    // the Android front end's first image of this renderer's scene and camera (DrawView.cpp:47-210
    // arrays drawn by MainRenderer.copyFrame, MainRenderer.java:338-546): flat-coloured triangles,
    // back faces culled, nearest surface kept, background 0, same bitmap format as renderFrame
    void rasterPreview(std::uint32_t *bitmap, std::uint32_t stride) noexcept;

    // extensions: stream key, Russian-roulette depths, last failure
    void setSeed(std::uint64_t seed) noexcept { seed_ = seed; }
    void setDepths(std::int32_t depthMin, std::int32_t depthMax) noexcept { depthMin_ = depthMin; depthMax_ = depthMax; }
    const std::string &lastError() const noexcept { return error_; }

private:
    std::unique_ptr<Sampler> samplerPixel_{};
    std::uint32_t width_{}, height_{}, samplesPixel_{};
    std::uint64_t seed_{0};
    std::int32_t depthMin_{RayDepthMin}, depthMax_{RayDepthMax};
    std::string error_{};
};

}  // namespace MobileRT

namespace Components {

// Perspective.hpp:12-43
class Perspective final : public ::MobileRT::Camera {
public:
    explicit Perspective(const ::glm::vec3 &position, const ::glm::vec3 &lookAt, const ::glm::vec3 &up, float hFov,
                         float vFov) noexcept
        : Camera{position, lookAt, up}, hFov_{hFov}, vFov_{vFov} {}
    int kind() const noexcept final { return 0; }
    float hFovDegrees() const noexcept final { return hFov_; }
    float vFovDegrees() const noexcept final { return vFov_; }
    float getHFov() const noexcept { return hFov_; }
    float getVFov() const noexcept { return vFov_; }

private:
    float hFov_{}, vFov_{};
};

// Orthographic.hpp:12-45
class Orthographic final : public ::MobileRT::Camera {
public:
    explicit Orthographic(const ::glm::vec3 &position, const ::glm::vec3 &lookAt, const ::glm::vec3 &up, float sizeH,
                          float sizeV) noexcept
        : Camera{position, lookAt, up}, sizeH_{sizeH}, sizeV_{sizeV} {}
    int kind() const noexcept final { return 1; }
    float hFovDegrees() const noexcept final { return sizeH_; }   // the film size, for the C ABI
    float vFovDegrees() const noexcept final { return sizeV_; }
    float getSizeH() const noexcept { return sizeH_ / 2.0f; }     // the reference keeps half the size
    float getSizeV() const noexcept { return sizeV_ / 2.0f; }

private:
    float sizeH_{}, sizeV_{};
};

// Constant.hpp, Stratified.hpp, HaltonSeq.hpp, MersenneTwister.hpp
class Constant final : public ::MobileRT::Sampler {
public:
    explicit Constant(float value) noexcept : Sampler{CONSTANT, value} {}
};
class Stratified final : public ::MobileRT::Sampler {
public:
    explicit Stratified() noexcept : Sampler{STRATIFIED} {}
    explicit Stratified(std::uint32_t, std::uint32_t, std::uint32_t) noexcept : Sampler{STRATIFIED} {}
};
class HaltonSeq final : public ::MobileRT::Sampler {
public:
    explicit HaltonSeq() noexcept : Sampler{HALTON} {}
    explicit HaltonSeq(std::uint32_t, std::uint32_t, std::uint32_t) noexcept : Sampler{HALTON} {}
};
class MersenneTwister final : public ::MobileRT::Sampler {
public:
    explicit MersenneTwister() noexcept : Sampler{RANDOM} {}
};

// PointLight.hpp, AreaLight.hpp
class PointLight final : public ::MobileRT::Light {
public:
    ::MobileRT::detail::F3 position_{};
    explicit PointLight(const ::MobileRT::Material &radiance, const ::glm::vec3 &position) noexcept
        : Light{radiance}, position_{::MobileRT::detail::f3(position)} {}
    bool isArea() const noexcept final { return false; }
};
class AreaLight final : public ::MobileRT::Light {
public:
    ::MobileRT::detail::F3 a_{}, b_{}, c_{};
    std::unique_ptr<::MobileRT::Sampler> samplerPointLight_{};
    explicit AreaLight(const ::MobileRT::Material &radiance, std::unique_ptr<::MobileRT::Sampler> samplerPointLight,
                       const ::glm::vec3 &pointA, const ::glm::vec3 &pointB, const ::glm::vec3 &pointC) noexcept
        : Light{radiance}, a_{::MobileRT::detail::f3(pointA)}, b_{::MobileRT::detail::f3(pointB)},
          c_{::MobileRT::detail::f3(pointC)}, samplerPointLight_{std::move(samplerPointLight)} {}
    bool isArea() const noexcept final { return true; }
};

// NoShadows.hpp, Whitted.hpp, PathTracer.hpp
class NoShadows final : public ::MobileRT::Shader {
public:
    explicit NoShadows(::MobileRT::Scene &&scene, std::uint32_t samplesLight, Accelerator accelerator) noexcept
        : Shader{std::move(scene), samplesLight, accelerator} {}
    int shaderKind() const noexcept final { return 0; }
};
class Whitted final : public ::MobileRT::Shader {
public:
    explicit Whitted(::MobileRT::Scene &&scene, std::uint32_t samplesLight, Accelerator accelerator) noexcept
        : Shader{std::move(scene), samplesLight, accelerator} {}
    int shaderKind() const noexcept final { return 1; }
};
class PathTracer final : public ::MobileRT::Shader {
public:
    explicit PathTracer(::MobileRT::Scene &&scene, std::unique_ptr<::MobileRT::Sampler> samplerRussianRoulette,
                        std::uint32_t samplesLight, Accelerator accelerator) noexcept
        : Shader{std::move(scene), samplesLight, accelerator}, samplerRussianRoulette_{std::move(samplerRussianRoulette)} {}
    int shaderKind() const noexcept final { return 2; }
    const ::MobileRT::Sampler *russianRoulette() const noexcept final { return samplerRussianRoulette_.get(); }

private:
    std::unique_ptr<::MobileRT::Sampler> samplerRussianRoulette_{};
};

// DepthMap.hpp, DiffuseMaterial.hpp
class DepthMap final : public ::MobileRT::Shader {
public:
    explicit DepthMap(::MobileRT::Scene &&scene, const ::glm::vec3 &maxPoint, Accelerator accelerator) noexcept
        : Shader{std::move(scene), 0, accelerator}, maxPoint_{::MobileRT::detail::f3(maxPoint)} {}
    int shaderKind() const noexcept final { return 3; }
    ::MobileRT::detail::F3 depthPoint() const noexcept final { return maxPoint_; }

private:
    ::MobileRT::detail::F3 maxPoint_{};
};
class DiffuseMaterial final : public ::MobileRT::Shader {
public:
    explicit DiffuseMaterial(::MobileRT::Scene &&scene, Accelerator accelerator) noexcept
        : Shader{std::move(scene), 0, accelerator} {}
    int shaderKind() const noexcept final { return 4; }
};

// OBJLoader.hpp: reads a Wavefront OBJ and the named MTL file with the reference loader's conventions
// (OBJLoader.cpp:21-248) through the library's parser (mrt_obj_load).
class OBJLoader final {
public:
    explicit OBJLoader(std::string obj, std::string materials) noexcept;
    OBJLoader(const OBJLoader &) = delete;
    OBJLoader &operator=(const OBJLoader &) = delete;
    ~OBJLoader() noexcept;
    // number of triangles (emitting faces included), -1 when the files cannot be read
    std::int32_t process() noexcept;
    // appends the triangles, materials and area lights (each light sampler from `lambda`)
    bool fillScene(::MobileRT::Scene *scene, std::function<std::unique_ptr<::MobileRT::Sampler>()> lambda) noexcept;
    bool isProcessed() const noexcept { return isProcessed_; }
    const std::string &lastError() const noexcept { return error_; }

private:
    std::string objFilePath_{}, mtlFilePath_{};
    void *data_{nullptr};
    bool isProcessed_{false};
    std::int32_t numberTriangles_{-1};
    std::string error_{};
};

}  // namespace Components

#endif  // MRT_B200_API_HPP
