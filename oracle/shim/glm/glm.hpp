// Minimal stand-in for the subset of the GLM vector API that MobileRT's render path uses.
//
// Test infrastructure only: this header lets the reference sources compile here so they can act as
// the checker for the CUDA path.  The real GLM submodule is an empty directory in the reference
// checkout (app/third_party/glm, .gitmodules:1-6, no pinned commit), so its exact float bits cannot
// be reproduced; every function below is written from the GLSL 4.60 specification's definition of
// the built-in, with one fixed evaluation order.  The CUDA kernels use the same order, so parity is
// pinned to this header.
//
//   dot(a,b)        = (a.x*b.x + a.y*b.y) + a.z*b.z
//   cross(a,b)      = (a.y*b.z - b.y*a.z, a.z*b.x - b.z*a.x, a.x*b.y - b.x*a.y)
//   length(v)       = sqrt(dot(v,v))
//   normalize(v)    = v * (1 / sqrt(dot(v,v)))            (two roundings, never an rsqrt)
//   reflect(I,N)    = I - (N * dot(N,I)) * 2
//   refract(I,N,e)  = k = 1 - (e*e) * (1 - d*d); k < 0 ? 0 : e*I - (e*d + sqrt(k)) * N,  d = dot(N,I)
//   min(a,b)        = (b < a) ? b : a     max(a,b) = (a < b) ? b : a   (std::min / std::max rules)
#ifndef MRT_ORACLE_SHIM_GLM_HPP
#define MRT_ORACLE_SHIM_GLM_HPP

#include <cmath>
#include <cstdint>

namespace glm {

struct bvec3 {
    bool x, y, z;
};

struct vec3 {
    float x, y, z;

    constexpr vec3() noexcept : x(0.0f), y(0.0f), z(0.0f) {}
    constexpr explicit vec3(float s) noexcept : x(s), y(s), z(s) {}
    constexpr vec3(float a, float b, float c) noexcept : x(a), y(b), z(c) {}

    float &operator[](int i) noexcept { return i == 0 ? x : (i == 1 ? y : z); }
    const float &operator[](int i) const noexcept { return i == 0 ? x : (i == 1 ? y : z); }

    vec3 &operator+=(const vec3 &o) noexcept { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
    vec3 &operator-=(const vec3 &o) noexcept { x = x - o.x; y = y - o.y; z = z - o.z; return *this; }
    vec3 &operator*=(const vec3 &o) noexcept { x = x * o.x; y = y * o.y; z = z * o.z; return *this; }
    vec3 &operator/=(const vec3 &o) noexcept { x = x / o.x; y = y / o.y; z = z / o.z; return *this; }

    // Scalar compound forms convert the scalar to float first (so `/= uint32_t` divides by float(n)).
    template <typename S> vec3 &operator*=(S s) noexcept {
        const float f = static_cast<float>(s);
        x = x * f; y = y * f; z = z * f; return *this;
    }
    template <typename S> vec3 &operator/=(S s) noexcept {
        const float f = static_cast<float>(s);
        x = x / f; y = y / f; z = z / f; return *this;
    }
};

inline vec3 operator+(const vec3 &a, const vec3 &b) noexcept { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3 &a, const vec3 &b) noexcept { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(const vec3 &a, const vec3 &b) noexcept { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator/(const vec3 &a, const vec3 &b) noexcept { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline vec3 operator-(const vec3 &a) noexcept { return vec3(-a.x, -a.y, -a.z); }

inline vec3 operator+(const vec3 &a, float s) noexcept { return vec3(a.x + s, a.y + s, a.z + s); }
inline vec3 operator-(const vec3 &a, float s) noexcept { return vec3(a.x - s, a.y - s, a.z - s); }
inline vec3 operator*(const vec3 &a, float s) noexcept { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator/(const vec3 &a, float s) noexcept { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec3 operator+(float s, const vec3 &a) noexcept { return vec3(s + a.x, s + a.y, s + a.z); }
inline vec3 operator-(float s, const vec3 &a) noexcept { return vec3(s - a.x, s - a.y, s - a.z); }
inline vec3 operator*(float s, const vec3 &a) noexcept { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(float s, const vec3 &a) noexcept { return vec3(s / a.x, s / a.y, s / a.z); }

inline float dot(const vec3 &a, const vec3 &b) noexcept {
    const float px = a.x * b.x;
    const float py = a.y * b.y;
    const float pz = a.z * b.z;
    return (px + py) + pz;
}

inline vec3 cross(const vec3 &a, const vec3 &b) noexcept {
    return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

inline float length(const vec3 &v) noexcept { return std::sqrt(dot(v, v)); }

inline vec3 normalize(const vec3 &v) noexcept {
    const float inv = 1.0f / std::sqrt(dot(v, v));
    return v * inv;
}

inline vec3 reflect(const vec3 &i, const vec3 &n) noexcept {
    const float d = dot(n, i);
    return i - (n * d) * 2.0f;
}

inline vec3 refract(const vec3 &i, const vec3 &n, float eta) noexcept {
    const float d = dot(n, i);
    const float k = 1.0f - (eta * eta) * (1.0f - d * d);
    if (k < 0.0f) {
        return vec3(0.0f);
    }
    const float s = eta * d + std::sqrt(k);
    return (eta * i) - (s * n);
}

inline float min(float a, float b) noexcept { return (b < a) ? b : a; }
inline float max(float a, float b) noexcept { return (a < b) ? b : a; }
inline vec3 min(const vec3 &a, const vec3 &b) noexcept {
    return vec3((b.x < a.x) ? b.x : a.x, (b.y < a.y) ? b.y : a.y, (b.z < a.z) ? b.z : a.z);
}
inline vec3 max(const vec3 &a, const vec3 &b) noexcept {
    return vec3((a.x < b.x) ? b.x : a.x, (a.y < b.y) ? b.y : a.y, (a.z < b.z) ? b.z : a.z);
}
inline vec3 abs(const vec3 &v) noexcept { return vec3(std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)); }

inline bvec3 greaterThan(const vec3 &a, const vec3 &b) noexcept { return bvec3{a.x > b.x, a.y > b.y, a.z > b.z}; }
inline bvec3 lessThanEqual(const vec3 &a, const vec3 &b) noexcept { return bvec3{a.x <= b.x, a.y <= b.y, a.z <= b.z}; }
inline bool any(const bvec3 &b) noexcept { return b.x || b.y || b.z; }
inline bool all(const bvec3 &b) noexcept { return b.x && b.y && b.z; }

}  // namespace glm

#endif  // MRT_ORACLE_SHIM_GLM_HPP
