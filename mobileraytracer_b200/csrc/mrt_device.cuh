// mrt_device.cuh - device arithmetic of the MobileRT render path.
//
// Every function keeps the float operation order of the reference source it cites (files of the
// MobileRayTracer checkout, app/...).  The library is compiled with --fmad=false -prec-div=true
// -prec-sqrt=true (no FMA contraction, IEEE division and square root, denormals kept), so these
// expressions round exactly as the reference's compiled C++ does.  GLM built-ins follow the fixed
// evaluation order documented in the oracle's glm stand-in:
//   dot = (x*x' + y*y') + z*z',  normalize(v) = v * (1/sqrt(dot(v,v))),
//   std::min(a,b) = (b < a) ? b : a,  std::max(a,b) = (a < b) ? b : a.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/mrt_cuda.h"

namespace mrt {

constexpr float kEpsilon = 1.0e-06f;        // Utils.hpp:37
constexpr float kRayLengthMax = 1.0e+30f;   // Utils.hpp:33
constexpr int kWide = 8;                    // children per node of the FAST tree
constexpr int kNodeWords = 32;              // 32-bit words per node of the FAST tree (128 bytes)
// Word positions in a FAST node.  Each 64-byte half holds what the test of four children reads: the
// first the grid origin (words 0-2), the grid exponents and internal-child mask (3) and the planes of
// slots 0-3, the second the first internal child's node index (16), the first leaf triangle's record
// index (17), the leaf meta bytes of slots 0-3 and 4-7 (18, 19) and the planes of slots 4-7.
constexpr int kNodeChildBase = 16, kNodeTriBase = 17, kNodeMeta = 18;
__host__ __device__ constexpr int node_plane_word(int axis, int slot) { return (slot < 4 ? 4 : 20) + 4 * axis + (slot & 3); }
constexpr uint32_t kMaxLeafTris = 3;        // triangles per leaf child of the FAST tree
constexpr uint32_t kMaxFastTris = 1u << 27; // triangles of one FAST tree (indices and counts stay in 32 bits)
constexpr float kSphereEpsilon = 1.0e-05f;  // Sphere.cpp:43,50

#define MRT_HD __host__ __device__ __forceinline__

struct V3 {
    float x, y, z;
};
MRT_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
MRT_HD V3 v3(float4 f) { return V3{f.x, f.y, f.z}; }
MRT_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
MRT_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
MRT_HD V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
MRT_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
MRT_HD V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
MRT_HD V3 adds(V3 a, float s) { return V3{a.x + s, a.y + s, a.z + s}; }
MRT_HD V3 subs(V3 a, float s) { return V3{a.x - s, a.y - s, a.z - s}; }
MRT_HD float dot(V3 a, V3 b) {
    const float px = a.x * b.x, py = a.y * b.y, pz = a.z * b.z;
    return (px + py) + pz;
}
MRT_HD V3 cross(V3 a, V3 b) { return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
MRT_HD float length(V3 v) { return sqrtf(dot(v, v)); }
MRT_HD V3 normalize(V3 v) {
    const float inv = 1.0f / sqrtf(dot(v, v));
    return v * inv;
}
MRT_HD float smin(float a, float b) { return (b < a) ? b : a; }
MRT_HD float smax(float a, float b) { return (a < b) ? b : a; }
MRT_HD V3 vmin(V3 a, V3 b) { return V3{smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)}; }
MRT_HD V3 vmax(V3 a, V3 b) { return V3{smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)}; }
MRT_HD bool any_pos(V3 a) { return a.x > 0.0f || a.y > 0.0f || a.z > 0.0f; }
MRT_HD float comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
// glm::reflect(I, N) = I - (N * dot(N, I)) * 2
MRT_HD V3 reflect(V3 i, V3 n) {
    const float d = dot(n, i);
    return i - (n * d) * 2.0f;
}
// glm::refract(I, N, eta), GLSL definition
MRT_HD V3 refract(V3 i, V3 n, float eta) {
    const float d = dot(n, i);
    const float k = 1.0f - (eta * eta) * (1.0f - d * d);
    if (k < 0.0f) return V3{0.0f, 0.0f, 0.0f};
    const float s = eta * d + sqrtf(k);
    return V3{eta * i.x, eta * i.y, eta * i.z} - V3{s * n.x, s * n.y, s * n.z};
}

// float -> int32 / uint32 as the reference build converts on x86-64 (cvttss2si): out-of-range and
// NaN give INT32_MIN for int32; uint32 goes through a 64-bit signed register and keeps the low
// 32 bits (NaN / out of range: 0).  CUDA's own conversions saturate instead.
MRT_HD int32_t f2i_x86(float f) {
    if (!(f > -2147483904.0f && f < 2147483648.0f)) return INT32_MIN;
    return (int32_t)f;
}
MRT_HD uint32_t f2u_x86(float f) {
    if (!(f > -9.2233720368547758e18f && f < 9.2233720368547758e18f)) return 0u;
    return (uint32_t)(int64_t)f;
}

struct Box {
    V3 mn, mx;
};

// ---------------------------------------------------------------------------------------------
// Device scene
// ---------------------------------------------------------------------------------------------
struct DevMaterial {
    V3 le, kd, ks, kt;
    float ior;
};

struct DevLight {
    int32_t kind;
    V3 pos;             // point light
    V3 a, ab, ac;       // area light triangle (AreaLight.cpp:13-19: Triangle{A, B, C, -1})
    V3 na;              // its computed normal (unused by the shaders, kept for completeness)
    DevMaterial radiance;
};

// reference BVH node (BVH.hpp:21-25): AABB + indexOffset_ + numberPrimitives_
struct RefNode {
    float mn[3];
    float mx[3];
    uint32_t offset;
    uint32_t count;
};

struct DevGrid {
    int32_t G;
    uint32_t shift;
    int32_t index_mode;
    int32_t has;
    V3 mn, mx;          // m_Extends
    V3 sr, cw;          // m_SR, m_CW
    const uint32_t *start;  // G^3 + 1
    const uint32_t *refs;
    const float *trec;      // triangle grid: 16 floats per triangle in input order (A, AB, AC, 7 unused),
                            // 64-byte aligned records the walk reads with one 256-bit and one 32-bit load
};

enum PrimType { kPlane = 0, kSphere = 1, kTriangle = 2 };

struct DevScene {
    uint32_t n_tri, n_sph, n_pln, n_light, n_mat;
    // triangles in input order: A, AB, AC (Triangle.hpp:16-18), shading data
    const float4 *tri_a;
    const float4 *tri_ab;
    const float4 *tri_ac;
    const float *tri_n;    // 9 per triangle
    const float *tri_c;    // 9 per triangle
    const int32_t *tri_mat;
    const float4 *sph;     // center, sq_radius
    const int32_t *sph_mat;
    const float4 *pln_n;   // normalised normal
    const float4 *pln_p;   // point
    const int32_t *pln_mat;
    const DevLight *lights;
    const DevMaterial *mats;
    // accelerators
    int32_t accel;
    int32_t bvh_mode;
    const float4 *fnodes;  // FAST BVH: 8-wide quantised nodes of 128 bytes (layout in mrt_trace.cuh)
    const float4 *ftris;   // FAST BVH: 3 float4 per triangle in leaf order (A|index, AB, AC)
    uint32_t n_fnodes;     // nodes in fnodes (bounds of every node index read)
    const RefNode *rnodes[3];
    uint32_t rnode_count[3];
    DevGrid grid[3];
    int32_t *error_flag;   // MRT_ERR_LIMIT when a traversal cap is hit
};

// ---------------------------------------------------------------------------------------------
// primitive tests
// ---------------------------------------------------------------------------------------------
struct Ray {
    V3 o, d;
    int32_t depth;
    uint32_t exclude;
};

// Triangle::intersect(Intersection*, Ray) up to the distance test, Triangle.cpp:57-86.
// Returns true and t/u/v when the hit passes the u, v and Epsilon tests (the caller applies the
// `t >= length` rejection so ties can be resolved by index).
MRT_HD bool tri_test(V3 a, V3 ab, V3 ac, const Ray &r, float &t, float &u, float &v) {
    const V3 perp = cross(r.d, ac);
    const float np = dot(ab, perp);
    if (fabsf(np) < kEpsilon) return false;
    const float inv = 1.0f / np;
    const V3 vtc = r.o - a;
    u = inv * dot(vtc, perp);
    if (u < 0.0f || u > 1.0f) return false;
    const V3 upp = cross(vtc, ab);
    v = inv * dot(r.d, upp);
    if (v < 0.0f || (u + v) > 1.0f) return false;
    t = inv * dot(ac, upp);
    if (t < kEpsilon) return false;
    return true;
}

// Triangle::intersect(Ray, dist), Triangle.cpp:105-136
MRT_HD bool tri_occ(V3 a, V3 ab, V3 ac, const Ray &r, float dist) {
    const V3 perp = cross(r.d, ac);
    const float np = dot(ab, perp);
    if (fabsf(np) < kEpsilon) return false;
    const float inv = 1.0f / np;
    const V3 vtc = r.o - a;
    const float u = inv * dot(vtc, perp);
    if (u < 0.0f || u > 1.0f) return false;
    const V3 upp = cross(vtc, ab);
    const float v = inv * dot(r.d, upp);
    if (v < 0.0f || (u + v) > 1.0f) return false;
    const float d = inv * dot(ac, upp);
    return d > kEpsilon && d < dist;
}

// quadratic of Sphere::intersect, Sphere.cpp:18-41
MRT_HD bool sph_solve(V3 center, float sq_radius, const Ray &r, float &t) {
    const V3 oc = center - r.o;
    const float proj = dot(oc, r.d);
    const float ocm = length(oc);
    const float A = dot(r.d, r.d);
    const float B = 2.0f * -proj;
    const float C = ocm * ocm - sq_radius;
    const float disc = B * B - 4.0f * A * C;
    if (disc < 0.0f) return false;
    const float root = sqrtf(disc);
    const float d1 = -B + root, d2 = -B - root;
    t = smin(d1, d2) / (2.0f * A);
    return true;
}

// Plane::intersect distance, Plane.cpp:17-34
MRT_HD bool pln_solve(V3 n, V3 p, const Ray &r, float &t) {
    const float np = dot(n, r.d);
    if (fabsf(np) < kEpsilon) return false;
    const V3 vtp = p - r.o;
    const float sp = dot(n, vtp);
    t = sp / np;
    return true;
}

// intersect(AABB, Ray), AABB.cpp:15-35
MRT_HD bool ref_box_hit(const float *mn, const float *mx, const Ray &r) {
    const float invx = 1.0f / r.d.x;
    const float t1x = (mn[0] - r.o.x) * invx;
    const float t2x = (mx[0] - r.o.x) * invx;
    float tmin = smin(t1x, t2x);
    float tmax = smax(t1x, t2x);
    {
        const float inv = 1.0f / r.d.y;
        const float t1 = (mn[1] - r.o.y) * inv;
        const float t2 = (mx[1] - r.o.y) * inv;
        tmin = smax(tmin, smin(t1, t2));
        tmax = smin(tmax, smax(t1, t2));
    }
    {
        const float inv = 1.0f / r.d.z;
        const float t1 = (mn[2] - r.o.z) * inv;
        const float t2 = (mx[2] - r.o.z) * inv;
        tmin = smax(tmin, smin(t1, t2));
        tmax = smin(tmax, smax(t1, t2));
    }
    return tmax >= smax(tmin, 0.0f);
}

// ---------------------------------------------------------------------------------------------
// keyed stream (the same definition as the oracle's): lowbias32 mixer (Wellons, hash-prospector)
// ---------------------------------------------------------------------------------------------
MRT_HD uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x21f0aaadu;
    x ^= x >> 15;
    x *= 0x735a2d97u;
    x ^= x >> 15;
    return x;
}
MRT_HD uint32_t key_base(uint64_t seed, uint32_t pixel, uint32_t sample) {
    uint32_t h = mix32((uint32_t)seed ^ 0x9e3779b9u);
    h = mix32(h ^ (uint32_t)(seed >> 32));
    h = mix32(h ^ pixel);
    return mix32(h ^ sample);
}
MRT_HD float key_float(uint32_t base, uint32_t node, uint32_t dim) {
    const uint32_t h = mix32(mix32(base ^ node) ^ dim);
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

// haltonSequence, Utils.cpp:36-45
MRT_HD float halton(uint32_t index, uint32_t base) {
    float f = 1.0f, result = 0.0f;
    while (index > 0) {
        f /= (float)base;
        result += f * (float)(index % base);
        index = index / base;
    }
    return result;
}

// Halton base of sample dimension `dim`: the dim-th prime.  The dimensions in use are 0-1 (camera
// jitter), 2 (roulette) and 8 + 3j + 1, 8 + 3j + 2 (position on the light of light sample j < 32),
// all below kHaltonDims, so no two dimensions share a base.
constexpr uint32_t kHaltonDims = 128;
#define MRT_HALTON_PRIMES \
    2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, \
    59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127, 131, \
    137, 139, 149, 151, 157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223, \
    227, 229, 233, 239, 241, 251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311, \
    313, 317, 331, 337, 347, 349, 353, 359, 367, 373, 379, 383, 389, 397, 401, 409, \
    419, 421, 431, 433, 439, 443, 449, 457, 461, 463, 467, 479, 487, 491, 499, 503, \
    509, 521, 523, 541, 547, 557, 563, 569, 571, 577, 587, 593, 599, 601, 607, 613, \
    617, 619, 631, 641, 643, 647, 653, 659, 661, 673, 677, 683, 691, 701, 709, 719
#ifdef __CUDACC__
static __constant__ uint32_t c_halton_primes[kHaltonDims] = {MRT_HALTON_PRIMES};
#endif
static const uint32_t h_halton_primes[kHaltonDims] = {MRT_HALTON_PRIMES};
MRT_HD uint32_t halton_base(uint32_t dim) {
#ifdef __CUDA_ARCH__
    return c_halton_primes[dim % kHaltonDims];
#else
    return h_halton_primes[dim % kHaltonDims];
#endif
}

struct Stream {
    uint64_t seed;
    uint32_t base;      // key_base(seed, pixel, sample)
    uint32_t rot_base;  // key_base(seed, pixel, 0xFFFFFFFF)
    uint32_t sample;
    uint32_t spp;
    float constant_value;
};

MRT_HD Stream make_stream(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t spp, float cval) {
    Stream s;
    s.seed = seed;
    s.base = key_base(seed, pixel, sample);
    s.rot_base = key_base(seed, pixel, 0xFFFFFFFFu);
    s.sample = sample;
    s.spp = spp;
    s.constant_value = cval;
    return s;
}

MRT_HD float draw(const Stream &st, int kind, uint32_t node, uint32_t dim) {
    switch (kind) {
        case MRT_SAMPLER_CONSTANT: return st.constant_value;
        case MRT_SAMPLER_STRATIFIED: {
            float v = (float)st.sample / (float)(st.spp > 0 ? st.spp : 1u) + key_float(st.rot_base, node, dim);
            if (v >= 1.0f) v -= 1.0f;
            return v;
        }
        case MRT_SAMPLER_HALTON: {
            float v = halton(st.sample, halton_base(dim)) + key_float(st.rot_base, node, dim);
            if (v >= 1.0f) v -= 1.0f;
            return v;
        }
        default: return key_float(st.base, node, dim);
    }
}

constexpr uint32_t kDimRR = 2u;
constexpr uint32_t kDimHemi = 3u;
constexpr uint32_t kDimLight = 8u;

// sin / cos of x in [0, 2*pi): quadrant reduction with a two-part pi/2 (Cody-Waite) and Taylor
// polynomials of degree 9 (sin) and 10 (cos) on [-pi/4, pi/4]; float multiplies and adds only
// (the same steps as the oracle), replacing std::sin / std::cos of Shader.cpp:217-219.
MRT_HD void sincos_turn(float x, float &s_out, float &c_out) {
    const float two_over_pi = 0.636619772367581343f;
    const float pio2_hi = 1.5703125f;
    const float pio2_lo = 4.83826794897e-4f;
    float kf = x * two_over_pi + 0.5f;
    const int32_t k = (int32_t)kf;
    kf = (float)k;
    const float r = (x - kf * pio2_hi) - kf * pio2_lo;
    const float r2 = r * r;
    const float sp = r + r * r2 * (-1.0f / 6.0f + r2 * (1.0f / 120.0f + r2 * (-1.0f / 5040.0f + r2 * (1.0f / 362880.0f))));
    const float cp = 1.0f + r2 * (-0.5f + r2 * (1.0f / 24.0f + r2 * (-1.0f / 720.0f + r2 * (1.0f / 40320.0f + r2 * (-1.0f / 3628800.0f)))));
    switch (k & 3) {
        case 0: s_out = sp; c_out = cp; break;
        case 1: s_out = cp; c_out = -sp; break;
        case 2: s_out = -sp; c_out = -cp; break;
        default: s_out = -cp; c_out = sp; break;
    }
}

// Shader::getCosineSampleHemisphere, Shader.cpp:193-223
MRT_HD V3 hemisphere(V3 n, float u1, float u2) {
    const float phi = 6.28318530717958647692f * u1;
    const float r2 = u2;
    const float cos_theta = sqrtf(r2);
    V3 u = fabsf(n.x) > 0.1f ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
    u = normalize(cross(u, n));
    const V3 v = cross(n, u);
    float sp, cp;
    sincos_turn(phi, sp, cp);
    const V3 dir = (u * (cp * cos_theta) + v * (sp * cos_theta)) + n * sqrtf(1.0f - r2);
    return normalize(dir);
}

// ---------------------------------------------------------------------------------------------
// camera: Camera.cpp:52-57 (basis), Perspective.cpp:10-44
// ---------------------------------------------------------------------------------------------
struct DevCamera {
    V3 position, direction, right, up;
    float hfov, vfov;   // Perspective: field of view in radians; Orthographic: half film size
    int32_t kind;       // MRT_CAMERA_*
};

MRT_HD float fast_arctan(float x) {
    const float ax = fabsf(x);
    return 0.785398163397448309616f * x - (x * (ax - 1.0f)) * (0.2447f + (0.0663f * ax));
}

MRT_HD Ray camera_ray(const DevCamera &k, float u, float v, float du, float dv) {
    if (k.kind == MRT_CAMERA_ORTHOGRAPHIC) {   // Orthographic::generateRay, Orthographic.cpp:23-34
        const float rf = (u - 0.5f) * k.hfov;
        const V3 right = k.right * rf + k.right * du;
        const float uf = (0.5f - v) * k.vfov;
        const V3 up = k.up * uf + k.up * dv;
        Ray r;
        r.d = k.direction;
        r.o = (k.position + right) + up;
        r.depth = 1;
        r.exclude = MRT_HIT_NONE;
        return r;
    }
    const float rf = fast_arctan(k.hfov * (u - 0.5f)) + du;
    const V3 right = k.right * rf;
    const float uf = fast_arctan(k.vfov * (0.5f - v)) + dv;
    const V3 up = k.up * uf;
    const V3 dest = ((k.position + k.direction) + right) + up;
    Ray r;
    r.d = normalize(dest - k.position);
    r.o = k.position;
    r.depth = 1;
    r.exclude = MRT_HIT_NONE;
    return r;
}

// incrementalAvg, Utils.cpp:48-70
MRT_HD uint32_t incremental_avg(V3 c, uint32_t avg, uint32_t n) {
    const uint32_t lr = avg & 0xFFu, lg = (avg >> 8u) & 0xFFu, lb = (avg >> 16u) & 0xFFu;
    const uint32_t sr = f2u_x86(c.x * 255.0f), sg = f2u_x86(c.y * 255.0f), sb = f2u_x86(c.z * 255.0f);
    const uint32_t cr = ((n - 1u) * lr + sr) / n, cg = ((n - 1u) * lg + sg) / n, cb = ((n - 1u) * lb + sb) / n;
    const uint32_t rr = cr < 255u ? cr : 255u, rg = cg < 255u ? cg : 255u, rb = cb < 255u ? cb : 255u;
    return 0xFF000000u | (rb << 16u) | (rg << 8u) | rr;
}

}  // namespace mrt
