// Minimal glm::vec3 for building the drop-in without GLM installed.  Callers that use the real GLM
// put it first on their include path; the drop-in library only ever receives plain floats, so
// either definition works with it.  Provides storage, construction, indexing and + - * /.
#ifndef MRT_GLM_MIN_HPP
#define MRT_GLM_MIN_HPP
namespace glm {
struct vec3 {
    float x, y, z;
    constexpr vec3() noexcept : x(0.0f), y(0.0f), z(0.0f) {}
    constexpr explicit vec3(float s) noexcept : x(s), y(s), z(s) {}
    constexpr vec3(float a, float b, float c) noexcept : x(a), y(b), z(c) {}
    float &operator[](int i) noexcept { return i == 0 ? x : (i == 1 ? y : z); }
    const float &operator[](int i) const noexcept { return i == 0 ? x : (i == 1 ? y : z); }
};
inline vec3 operator+(const vec3 &a, const vec3 &b) noexcept { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3 &a, const vec3 &b) noexcept { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(const vec3 &a, float s) noexcept { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator/(const vec3 &a, float s) noexcept { return vec3(a.x / s, a.y / s, a.z / s); }
}  // namespace glm
#endif
