// mrt_raster.cu - raster preview: the scene's triangles drawn with flat colours and a depth test.
//
// Reference: when a render starts, the Android front end first draws the scene with OpenGL ES 2.0 and
// shows that image until the ray tracer's pixels replace it.  DrawView.cpp:118-210 (initVerticesArray,
// initColorsArray) hands MainRenderer the triangles as (A, A + AB, A + AC) with z negated and one
// colour per triangle; DrawView.cpp:47-102 (initCameraArray) the camera; MainRenderer.copyFrame
// (MainRenderer.java:338-546) builds the model (identity), view (Matrix.setLookAtM on the z-negated
// position, direction and up) and projection (Matrix.perspectiveM with fovY = 0.918 x the vertical
// field of view, aspect from the frame, near 0.1, far 1e38; Matrix.orthoM with the film half sizes for
// Orthographic), and draws GL_TRIANGLES with VertexShaderRaster.glsl (P * V * M * position) and
// FragmentShaderRaster.glsl (the vertex colour) under the state of onSurfaceCreated
// (MainRenderer.java:206-235: back faces culled, counter-clockwise front faces, depth test LEQUAL,
// depth cleared to 1, colour cleared to 0); copyFrameBuffer (MainRenderer.java:111-139) reads the
// RGBA framebuffer back with the rows flipped.
//
// Here the same pipeline runs as CUDA kernels.  The parts OpenGL leaves to the implementation are
// fixed as follows (the oracle restates exactly these):
//   * projection x view is formed once on the host (column-major products, terms in index order);
//     a vertex's clip coordinates are that matrix times (x, y, -z, 1), terms in index order;
//   * clipping against the near and far planes and a guard band of 16 viewports in x and y
//     (Sutherland-Hodgman, polygon fanned from its first vertex); the guard band only bounds the
//     integer arithmetic, it removes no pixel of the viewport;
//   * window coordinates snapped to 1/256 pixel (round to nearest even); coverage at pixel centres by
//     exact 64-bit edge functions with the top-left rule; zero-area and clockwise triangles dropped;
//   * depth interpolated linearly in window space from the snapped edge functions and clamped to
//     [0, 1]; depth test LEQUAL in draw order = the smallest depth wins, a later triangle wins a tie
//     (one 64-bit atomicMin of (depth bits, ~triangle index) per covered pixel);
//   * the fragment colour is the triangle's colour (all three vertices carry it), converted to 8 bits
//     by round(clamp(c, 0, 1) * 255).
// One thread sets up and clips each triangle and covers the pixels of small ones (bounding box of at
// most 64 pixels, the soups' case); larger ones go to a queue that a block per triangle covers.
#include <algorithm>
#include <cmath>

#include "mrt_internal.h"

using namespace mrt;
using namespace mrt_host;

namespace {

constexpr float kSub = 256.0f;            // snapped window coordinates: 1/256 pixel
constexpr float kGuard = 16.0f;           // x, y clipped to +-16 w
constexpr uint32_t kSmallPixels = 64;     // bounding boxes up to this many pixels: one thread
// a triangle clipped by six planes has at most 9 vertices in exact arithmetic; rounded intersection
// points can make the polygon slightly non-convex and let a later plane add more, so the clipper
// keeps room for 16 and drops any vertex beyond that (the oracle does the same)
constexpr int kMaxPoly = 16;
constexpr uint32_t kMaxSide = 8192;       // frame sides (keeps every snapped coordinate in 32 bits)

// column-major 4x4: element (row r, column c) at m[4 c + r], as android.opengl.Matrix
struct Mat4 {
    float m[16];
};

// Matrix.perspectiveM: f = 1 / tan(fovy * pi / 360) with the tangent in double precision
Mat4 perspective_m(float fovy, float aspect, float znear, float zfar) {
    Mat4 r{};
    const float f = 1.0f / (float)std::tan((double)fovy * (3.14159265358979323846 / 360.0));
    const float range_rcp = 1.0f / (znear - zfar);
    r.m[0] = f / aspect;
    r.m[5] = f;
    r.m[10] = (zfar + znear) * range_rcp;
    r.m[11] = -1.0f;
    r.m[14] = 2.0f * zfar * znear * range_rcp;
    return r;
}

// Matrix.orthoM
Mat4 ortho_m(float left, float right, float bottom, float top, float znear, float zfar) {
    Mat4 r{};
    const float rw = 1.0f / (right - left), rh = 1.0f / (top - bottom), rd = 1.0f / (zfar - znear);
    r.m[0] = 2.0f * rw;
    r.m[5] = 2.0f * rh;
    r.m[10] = -2.0f * rd;
    r.m[12] = -(right + left) * rw;
    r.m[13] = -(top + bottom) * rh;
    r.m[14] = -(zfar + znear) * rd;
    r.m[15] = 1.0f;
    return r;
}

// Matrix.length: the float sum of squares, square root rounded to float
float length3(float x, float y, float z) { return std::sqrt(x * x + y * y + z * z); }

// Matrix.setLookAtM: forward f, side s = f x up, u = s x f, rows (s, u, -f), then translateM by -eye
Mat4 look_at_m(float ex, float ey, float ez, float cx, float cy, float cz, float ux, float uy, float uz) {
    float fx = cx - ex, fy = cy - ey, fz = cz - ez;
    const float rlf = 1.0f / length3(fx, fy, fz);
    fx *= rlf; fy *= rlf; fz *= rlf;
    float sx = fy * uz - fz * uy, sy = fz * ux - fx * uz, sz = fx * uy - fy * ux;
    const float rls = 1.0f / length3(sx, sy, sz);
    sx *= rls; sy *= rls; sz *= rls;
    const float vx = sy * fz - sz * fy, vy = sz * fx - sx * fz, vz = sx * fy - sy * fx;
    Mat4 r{};
    r.m[0] = sx; r.m[1] = vx; r.m[2] = -fx;
    r.m[4] = sy; r.m[5] = vy; r.m[6] = -fy;
    r.m[8] = sz; r.m[9] = vz; r.m[10] = -fz;
    r.m[15] = 1.0f;
    for (int i = 0; i < 4; ++i) r.m[12 + i] += r.m[i] * -ex + r.m[4 + i] * -ey + r.m[8 + i] * -ez;
    return r;
}

// a x b, each element's four terms added in index order
Mat4 mul_mm(const Mat4 &a, const Mat4 &b) {
    Mat4 r{};
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            r.m[4 * c + row] = ((a.m[row] * b.m[4 * c] + a.m[4 + row] * b.m[4 * c + 1]) + a.m[8 + row] * b.m[4 * c + 2]) +
                               a.m[12 + row] * b.m[4 * c + 3];
    return r;
}

// projection x view of MainRenderer.copyFrame for this camera and frame (the model matrix is the
// identity).  Camera vectors as Camera.cpp computes them; radToDeg(degToRad(v)) as
// Perspective::getVFov returns the field of view; Orthographic::getSizeH/V return the half sizes.
Mat4 preview_matrix(const MrtCamera &cam, uint32_t width, uint32_t height) {
    const DevCamera k = make_camera(cam);
    const float ex = k.position.x, ey = k.position.y, ez = -k.position.z;
    const float dx = k.direction.x, dy = k.direction.y, dz = -k.direction.z;
    const float ux = k.up.x, uy = k.up.y, uz = -k.up.z;
    const float znear = 0.1f, zfar = 1.0e38f;
    Mat4 proj{};
    if (cam.kind == MRT_CAMERA_ORTHOGRAPHIC) {
        const float size_h = k.hfov, size_v = k.vfov;
        proj = ortho_m(-size_h / 2, size_h / 2, -size_v / 2, size_v / 2, znear, zfar);
    } else {
        const float pi = 3.14159265358979323846f;
        const float w = (float)width, h = (float)height;
        const float ratio = std::max(w / h, h / w);
        const float hfov_factor = width > height ? ratio : 1.0f;
        const float vfov_factor = width < height ? ratio : 1.0f;
        float fovy = (k.vfov / pi) * 180.0f;
        fovy *= 0.918f;
        const float aspect = hfov_factor > vfov_factor ? hfov_factor : 1.0f / vfov_factor;
        proj = perspective_m(fovy, aspect, znear, zfar);
    }
    const Mat4 view = look_at_m(ex, ey, ez, ex + dx, ey + dy, ez + dz, ux, uy, uz);
    return mul_mm(proj, view);
}

// ------------------------------------------------------------------------------------------------
struct RasterTri {         // a front-facing triangle whose bounding box exceeds kSmallPixels
    int32_t x[3], y[3];    // snapped window coordinates
    float z[3];            // window depth
    uint32_t tri;          // scene triangle (draw order)
    uint32_t x0, x1, y0, y1;   // pixel box inside the viewport
};

struct RasterParams {
    float m[16];                  // projection x view, column-major
    uint32_t width, height;
    unsigned long long *keys;     // width x height: (depth bits << 32) | (0xFFFFFFFF - triangle)
    RasterTri *big;
    uint32_t big_cap;
    unsigned long long *counts;   // [0] queued, [1] drawn, [2] fragments, [3] triangles sent to the next pass
    uint32_t *overflow;           // triangles whose large pieces found the queue full
};

constexpr uint32_t kEmptyQueued = 0xFFFFFFFFu;   // a queue slot left empty by a triangle sent to the next pass

struct Clip {
    float x, y, z, w;
};

__device__ __forceinline__ float plane_dist(const Clip &v, int p) {
    switch (p) {
        case 0: return v.z + v.w;              // near
        case 1: return v.w - v.z;              // far
        case 2: return kGuard * v.w - v.x;
        case 3: return kGuard * v.w + v.x;
        case 4: return kGuard * v.w - v.y;
        default: return kGuard * v.w + v.y;
    }
}

__device__ __forceinline__ Clip to_clip(const float *m, float x, float y, float z) {
    Clip c;
    c.x = ((m[0] * x + m[4] * y) + m[8] * z) + m[12];
    c.y = ((m[1] * x + m[5] * y) + m[9] * z) + m[13];
    c.z = ((m[2] * x + m[6] * y) + m[10] * z) + m[14];
    c.w = ((m[3] * x + m[7] * y) + m[11] * z) + m[15];
    return c;
}

__device__ __forceinline__ long long edge_fn(long long xa, long long ya, long long xb, long long yb, long long px,
                                             long long py) {
    return (xb - xa) * (py - ya) - (yb - ya) * (px - xa);
}

// an edge of a counter-clockwise triangle owns the pixel centres on it when it is a left edge
// (going down) or a top edge (horizontal, going left)
__device__ __forceinline__ bool top_left(int32_t xa, int32_t ya, int32_t xb, int32_t yb) {
    return yb < ya || (yb == ya && xb < xa);
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

__device__ __forceinline__ long long floor_div256(long long a) { return a >= 0 ? a / 256 : -((-a + 255) / 256); }

struct Setup {
    int32_t x[3], y[3];
    float z[3];
    long long area2;
    bool tl12, tl20, tl01;
    float inv_area;
};

__device__ __forceinline__ bool cover(const Setup &t, uint32_t px, uint32_t py, float &z) {
    const long long cx = (long long)px * 256 + 128, cy = (long long)py * 256 + 128;
    const long long w0 = edge_fn(t.x[1], t.y[1], t.x[2], t.y[2], cx, cy);
    const long long w1 = edge_fn(t.x[2], t.y[2], t.x[0], t.y[0], cx, cy);
    const long long w2 = edge_fn(t.x[0], t.y[0], t.x[1], t.y[1], cx, cy);
    if (!((w0 > 0 || (w0 == 0 && t.tl12)) && (w1 > 0 || (w1 == 0 && t.tl20)) && (w2 > 0 || (w2 == 0 && t.tl01))))
        return false;
    z = t.z[0] + ((float)w1 * (t.z[1] - t.z[0]) + (float)w2 * (t.z[2] - t.z[0])) * t.inv_area;
    if (!(z > 0.0f)) z = 0.0f;   // (never -0: the key compares depth bits)
    if (z > 1.0f) z = 1.0f;
    return true;
}

__device__ __forceinline__ unsigned long long depth_key(float z, uint32_t tri) {
    return ((unsigned long long)__float_as_uint(z) << 32) | (unsigned long long)(0xFFFFFFFFu - tri);
}

// the pixel centres of a box, edge functions stepped exactly from pixel to pixel
__device__ __forceinline__ unsigned long long cover_box(const RasterParams &p, const Setup &t, uint32_t tri, uint32_t x0,
                                                        uint32_t x1, uint32_t y0, uint32_t y1) {
    const long long cx = (long long)x0 * 256 + 128, cy = (long long)y0 * 256 + 128;
    long long r0 = edge_fn(t.x[1], t.y[1], t.x[2], t.y[2], cx, cy);
    long long r1 = edge_fn(t.x[2], t.y[2], t.x[0], t.y[0], cx, cy);
    long long r2 = edge_fn(t.x[0], t.y[0], t.x[1], t.y[1], cx, cy);
    const long long sx0 = -256ll * (t.y[2] - t.y[1]), sy0 = 256ll * (t.x[2] - t.x[1]);
    const long long sx1 = -256ll * (t.y[0] - t.y[2]), sy1 = 256ll * (t.x[0] - t.x[2]);
    const long long sx2 = -256ll * (t.y[1] - t.y[0]), sy2 = 256ll * (t.x[1] - t.x[0]);
    unsigned long long n = 0;
    for (uint32_t py = y0; py <= y1; ++py, r0 += sy0, r1 += sy1, r2 += sy2) {
        long long w0 = r0, w1 = r1, w2 = r2;
        for (uint32_t px = x0; px <= x1; ++px, w0 += sx0, w1 += sx1, w2 += sx2) {
            if (!((w0 > 0 || (w0 == 0 && t.tl12)) && (w1 > 0 || (w1 == 0 && t.tl20)) && (w2 > 0 || (w2 == 0 && t.tl01))))
                continue;
            float z = t.z[0] + ((float)w1 * (t.z[1] - t.z[0]) + (float)w2 * (t.z[2] - t.z[0])) * t.inv_area;
            if (!(z > 0.0f)) z = 0.0f;
            if (z > 1.0f) z = 1.0f;
            atomicMin(&p.keys[(size_t)py * p.width + px], depth_key(z, tri));
            ++n;
        }
    }
    return n;
}

struct Win {        // a vertex in window coordinates
    int32_t x, y;   // snapped
    float z;
};

__device__ __forceinline__ Win to_window(const RasterParams &p, const Clip &c) {
    const float hw = 0.5f * (float)p.width, hh = 0.5f * (float)p.height;
    const float xn = c.x / c.w, yn = c.y / c.w, zn = c.z / c.w;
    return Win{__float2int_rn((hw * xn + hw) * kSub), __float2int_rn((hh * yn + hh) * kSub), 0.5f * zn + 0.5f};
}

// one triangle in window coordinates: back faces and empty boxes dropped (kind 0), boxes of up to
// kSmallPixels pixels covered here (kind 1), larger ones queued for k_raster_big (kind 2), front
// faces whose box misses the viewport counted as drawn only (kind 3)
struct SubTri {
    Setup t;
    int kind;
    uint32_t x0, x1, y0, y1;
};

__device__ __forceinline__ SubTri setup_sub(const RasterParams &p, Win a, Win b, Win c) {
    SubTri u;
    Setup &t = u.t;
    u.kind = 0;
    u.x0 = u.x1 = u.y0 = u.y1 = 0;
    t.x[0] = a.x; t.y[0] = a.y; t.z[0] = a.z;
    t.x[1] = b.x; t.y[1] = b.y; t.z[1] = b.z;
    t.x[2] = c.x; t.y[2] = c.y; t.z[2] = c.z;
    t.area2 = edge_fn(t.x[0], t.y[0], t.x[1], t.y[1], t.x[2], t.y[2]);
    if (t.area2 <= 0) return u;   // clockwise (back face, culled) or no area
    t.tl12 = top_left(t.x[1], t.y[1], t.x[2], t.y[2]);
    t.tl20 = top_left(t.x[2], t.y[2], t.x[0], t.y[0]);
    t.tl01 = top_left(t.x[0], t.y[0], t.x[1], t.y[1]);
    t.inv_area = 1.0f / (float)t.area2;
    const long long xmin = min(t.x[0], min(t.x[1], t.x[2])), xmax = max(t.x[0], max(t.x[1], t.x[2]));
    const long long ymin = min(t.y[0], min(t.y[1], t.y[2])), ymax = max(t.y[0], max(t.y[1], t.y[2]));
    const long long bx0 = max(0ll, -floor_div256(-(xmin - 128)));
    const long long bx1 = min((long long)p.width - 1, floor_div256(xmax - 128));
    const long long by0 = max(0ll, -floor_div256(-(ymin - 128)));
    const long long by1 = min((long long)p.height - 1, floor_div256(ymax - 128));
    if (bx0 > bx1 || by0 > by1) { u.kind = 3; return u; }   // drawn, nothing covered
    u.x0 = (uint32_t)bx0; u.x1 = (uint32_t)bx1; u.y0 = (uint32_t)by0; u.y1 = (uint32_t)by1;
    const uint64_t box = (uint64_t)(bx1 - bx0 + 1) * (uint64_t)(by1 - by0 + 1);
    u.kind = box > kSmallPixels ? 2 : 1;
    return u;
}

__device__ __forceinline__ void draw_sub(const RasterParams &p, uint32_t tri, const SubTri &u, uint32_t &qslot,
                                         unsigned long long &drawn, unsigned long long &frags) {
    if (u.kind == 0) return;
    ++drawn;
    if (u.kind == 3) return;
    if (u.kind == 2) {
        RasterTri r;
        for (int j = 0; j < 3; ++j) { r.x[j] = u.t.x[j]; r.y[j] = u.t.y[j]; r.z[j] = u.t.z[j]; }
        r.tri = tri;
        r.x0 = u.x0; r.x1 = u.x1; r.y0 = u.y0; r.y1 = u.y1;
        p.big[qslot++] = r;
        return;
    }
    frags += cover_box(p, u.t, tri, u.x0, u.x1, u.y0, u.y1);
}

// Queue slots for a triangle's `nbig` large pieces, all or none.  When the queue has no room the
// triangle goes whole to the overflow list (drawn by a later pass, which keeps the result: the depth
// test is an atomicMin of (depth, triangle) keys, the same in any order); slots it was handed below
// the queue's end are marked empty for k_raster_big.
__device__ __forceinline__ bool reserve(const RasterParams &p, uint32_t tri, uint32_t nbig, uint32_t &qslot) {
    if (nbig == 0) return true;
    const unsigned long long q = atomicAdd(&p.counts[0], (unsigned long long)nbig);
    if (q + nbig <= p.big_cap) { qslot = (uint32_t)q; return true; }
    for (unsigned long long k = q; k < p.big_cap; ++k) p.big[k].tri = kEmptyQueued;
    const unsigned long long o = atomicAdd(&p.counts[3], 1ull);
    p.overflow[o] = tri;   // o < triangles of this pass: each triangle is sent on at most once
    return false;
}

// a triangle that leaves the near/far planes or the guard band: Sutherland-Hodgman against the six
// planes in order, then the polygon fanned from its first vertex (out of line: rare, and its
// polygon arrays would cost the common path registers)
__device__ __noinline__ void draw_clipped(const RasterParams &p, uint32_t tri, Clip c0, Clip c1, Clip c2,
                                          unsigned long long &drawn, unsigned long long &frags) {
    Clip poly[kMaxPoly], tmp[kMaxPoly];
    poly[0] = c0; poly[1] = c1; poly[2] = c2;
    int n = 3;
    for (int q = 0; q < 6 && n >= 3; ++q) {
        int m = 0;
        for (int k = 0; k < n; ++k) {
            const Clip S = poly[k], E = poly[k + 1 < n ? k + 1 : 0];
            const float ds = plane_dist(S, q), de = plane_dist(E, q);
            if (ds >= 0.0f && m < kMaxPoly) tmp[m++] = S;
            if ((ds >= 0.0f) != (de >= 0.0f) && m < kMaxPoly) {
                const float t = ds / (ds - de);
                tmp[m++] = Clip{S.x + t * (E.x - S.x), S.y + t * (E.y - S.y), S.z + t * (E.z - S.z), S.w + t * (E.w - S.w)};
            }
        }
        n = m;
        for (int k = 0; k < n; ++k) poly[k] = tmp[k];
    }
    if (n < 3) return;
    Win w[kMaxPoly];
    for (int k = 0; k < n; ++k) w[k] = to_window(p, poly[k]);
    uint32_t nbig = 0;
    for (int k = 1; k + 1 < n; ++k) nbig += setup_sub(p, w[0], w[k], w[k + 1]).kind == 2 ? 1u : 0u;
    uint32_t qslot = 0;
    if (!reserve(p, tri, nbig, qslot)) return;
    for (int k = 1; k + 1 < n; ++k) draw_sub(p, tri, setup_sub(p, w[0], w[k], w[k + 1]), qslot, drawn, frags);
}

// one thread per triangle of the pass: all scene triangles, or the overflow list of the last pass
__global__ void __launch_bounds__(128, 8) k_raster_tris(DevScene s, RasterParams p, const uint32_t *list, uint32_t n_items) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long drawn = 0, frags = 0;
    if (i < n_items) {
        const uint32_t tri = list ? list[i] : i;
        const float4 a = s.tri_a[tri], ab = s.tri_ab[tri], ac = s.tri_ac[tri];
        // DrawView.cpp:131-154: A, A + AB, A + AC, z negated
        const Clip c0 = to_clip(p.m, a.x, a.y, -a.z);
        const Clip c1 = to_clip(p.m, a.x + ab.x, a.y + ab.y, -(a.z + ab.z));
        const Clip c2 = to_clip(p.m, a.x + ac.x, a.y + ac.y, -(a.z + ac.z));
        bool inside = true;
        for (int q = 0; q < 6; ++q)
            inside = inside && plane_dist(c0, q) >= 0.0f && plane_dist(c1, q) >= 0.0f && plane_dist(c2, q) >= 0.0f;
        if (inside) {
            const SubTri u = setup_sub(p, to_window(p, c0), to_window(p, c1), to_window(p, c2));
            uint32_t qslot = 0;
            if (reserve(p, tri, u.kind == 2 ? 1u : 0u, qslot)) draw_sub(p, tri, u, qslot, drawn, frags);
        } else {
            draw_clipped(p, tri, c0, c1, c2, drawn, frags);
        }
    }
    drawn = warp_sum(drawn);
    frags = warp_sum(frags);
    if ((threadIdx.x & 31) == 0) {
        if (drawn) atomicAdd(&p.counts[1], (unsigned long long)drawn);
        if (frags) atomicAdd(&p.counts[2], (unsigned long long)frags);
    }
}

// the queued triangles: a block per triangle, its threads over the pixel box
__global__ void __launch_bounds__(256) k_raster_big(RasterParams p) {
    const uint32_t n = (uint32_t)min(p.counts[0], (unsigned long long)p.big_cap);
    unsigned long long frags = 0;
    for (uint32_t b = blockIdx.x; b < n; b += gridDim.x) {
        const RasterTri r = p.big[b];
        if (r.tri == kEmptyQueued) continue;
        Setup t;
        for (int j = 0; j < 3; ++j) { t.x[j] = r.x[j]; t.y[j] = r.y[j]; t.z[j] = r.z[j]; }
        t.area2 = edge_fn(t.x[0], t.y[0], t.x[1], t.y[1], t.x[2], t.y[2]);
        t.tl12 = top_left(t.x[1], t.y[1], t.x[2], t.y[2]);
        t.tl20 = top_left(t.x[2], t.y[2], t.x[0], t.y[0]);
        t.tl01 = top_left(t.x[0], t.y[0], t.x[1], t.y[1]);
        t.inv_area = 1.0f / (float)t.area2;
        const uint32_t bw = r.x1 - r.x0 + 1, bh = r.y1 - r.y0 + 1;
        const uint64_t total = (uint64_t)bw * bh;
        for (uint64_t k = threadIdx.x; k < total; k += blockDim.x) {
            const uint32_t px = r.x0 + (uint32_t)(k % bw), py = r.y0 + (uint32_t)(k / bw);
            float z;
            if (!cover(t, px, py, z)) continue;
            atomicMin(&p.keys[(size_t)py * p.width + px], depth_key(z, r.tri));
            ++frags;
        }
    }
    frags = warp_sum(frags);
    if ((threadIdx.x & 31) == 0 && frags) atomicAdd(&p.counts[2], (unsigned long long)frags);
}

// DrawView.cpp:178-196: max(Kd, Ks, Kt, Le) per component (glm::max(x, y) = x < y ? y : x), or the
// mean of the vertex colours
__device__ __forceinline__ V3 preview_color(const DevScene &s, uint32_t i) {
    const int32_t m = s.tri_mat ? s.tri_mat[i] : -1;
    if (m >= 0 && (uint32_t)m < s.n_mat) {
        const DevMaterial &mt = s.mats[m];
        V3 c = mt.kd;
        c = V3{mt.ks.x < c.x ? c.x : mt.ks.x, mt.ks.y < c.y ? c.y : mt.ks.y, mt.ks.z < c.z ? c.z : mt.ks.z};
        c = V3{mt.kt.x < c.x ? c.x : mt.kt.x, mt.kt.y < c.y ? c.y : mt.kt.y, mt.kt.z < c.z ? c.z : mt.kt.z};
        c = V3{mt.le.x < c.x ? c.x : mt.le.x, mt.le.y < c.y ? c.y : mt.le.y, mt.le.z < c.z ? c.z : mt.le.z};
        return c;
    }
    const float *k = s.tri_c + 9 * (size_t)i;
    return V3{((k[0] + k[3]) + k[6]) / 3.0f, ((k[1] + k[4]) + k[7]) / 3.0f, ((k[2] + k[5]) + k[8]) / 3.0f};
}

__device__ __forceinline__ uint32_t unorm8(float c) { return (uint32_t)(fminf(fmaxf(c, 0.0f), 1.0f) * 255.0f + 0.5f); }

// copyFrameBuffer: framebuffer row y (from the bottom) becomes bitmap row height - 1 - y
__global__ void k_raster_resolve(DevScene s, RasterParams p, uint32_t *bitmap, uint32_t stride_px) {
    const size_t n = (size_t)p.width * p.height;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(i % p.width), y = (uint32_t)(i / p.width);
        const unsigned long long key = p.keys[i];
        uint32_t out = 0u;
        if (key != ~0ull) {
            const uint32_t tri = 0xFFFFFFFFu - (uint32_t)(key & 0xFFFFFFFFull);
            const V3 c = preview_color(s, tri);
            out = unorm8(c.x) | (unorm8(c.y) << 8) | (unorm8(c.z) << 16) | (255u << 24);
        }
        bitmap[(size_t)(p.height - 1 - y) * stride_px + x] = out;
    }
}

}  // namespace

extern "C" int mrt_raster_preview(MrtScene *s, const MrtCamera *cam, uint32_t width, uint32_t height, uint32_t *bitmap,
                                  uint32_t stride_bytes, uint32_t mem, MrtRasterStats *stats) {
    if (!s || !cam || !bitmap) return MRT_ERR_ARG;
    MrtContext *ctx = s->ctx;
    if (width == 0 || height == 0 || width > kMaxSide || height > kMaxSide || stride_bytes < 4u * width ||
        (stride_bytes & 3u) || (mem != MRT_MEM_HOST && mem != MRT_MEM_DEVICE) ||
        (cam->kind != MRT_CAMERA_PERSPECTIVE && cam->kind != MRT_CAMERA_ORTHOGRAPHIC) ||
        !(cam->fov_h_deg > 0.0f) || !(cam->fov_v_deg > 0.0f)) {
        set_error(ctx, "mrt_raster_preview: invalid arguments (sides 1..%u, row pitch >= 4 * width and a multiple of 4, "
                       "positive field of view or film size)", kMaxSide);
        return MRT_ERR_ARG;
    }
    if (mem == MRT_MEM_DEVICE && ((uintptr_t)bitmap & 3u)) {
        set_error(ctx, "mrt_raster_preview: the bitmap must be 4-byte aligned");
        return MRT_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t q = ctx->stream;
    const size_t pixels = (size_t)width * height;
    // queue room for every triangle of scenes up to 2^20 triangles (58 MB); beyond that, triangles
    // whose large pieces find the queue full are drawn by further passes over an overflow list (same
    // result).  MRT_RASTER_QUEUE_CAP lowers the room (tests force the further passes with it); it
    // stays at least kMaxPoly - 2, the pieces of one clipped triangle, so every pass draws something.
    uint32_t big_cap = std::min<uint32_t>(s->n_tri, 1u << 20) + 1024u;
    if (const char *e = getenv("MRT_RASTER_QUEUE_CAP")) {
        const long v = atol(e);
        if (v > 0 && (unsigned long)v < big_cap) big_cap = (uint32_t)v;
    }
    big_cap = std::max<uint32_t>(big_cap, (uint32_t)(kMaxPoly - 2));
    int st = ensure(ctx, ctx->raster[0], 8 * pixels);
    if (st == MRT_OK) st = ensure(ctx, ctx->raster[1], sizeof(RasterTri) * (size_t)big_cap);
    if (st == MRT_OK) st = ensure(ctx, ctx->raster[2], 4 * sizeof(unsigned long long));
    if (st == MRT_OK) st = ensure(ctx, ctx->raster[4], 2 * sizeof(uint32_t) * (size_t)std::max<uint32_t>(s->n_tri, 1u));
    const size_t bm_bytes = (size_t)stride_bytes * height;
    uint32_t *d_bitmap = bitmap;
    if (st == MRT_OK && mem == MRT_MEM_HOST) {
        st = ensure(ctx, ctx->raster[3], bm_bytes);
        d_bitmap = (uint32_t *)ctx->raster[3].ptr;
        // rows keep the caller's bytes between width and the pitch
        if (st == MRT_OK && stride_bytes != 4u * width)
            st = cuda_status(ctx, cudaMemcpyAsync(d_bitmap, bitmap, bm_bytes, cudaMemcpyHostToDevice, q), "bitmap in");
    }
    if (st != MRT_OK) return st;
    RasterParams p{};
    const Mat4 pv = preview_matrix(*cam, width, height);
    for (int k = 0; k < 16; ++k) p.m[k] = pv.m[k];
    p.width = width;
    p.height = height;
    p.keys = (unsigned long long *)ctx->raster[0].ptr;
    p.big = (RasterTri *)ctx->raster[1].ptr;
    p.big_cap = big_cap;
    p.counts = (unsigned long long *)ctx->raster[2].ptr;
    uint32_t *lists[2] = {(uint32_t *)ctx->raster[4].ptr, (uint32_t *)ctx->raster[4].ptr + std::max<uint32_t>(s->n_tri, 1u)};
    p.overflow = lists[0];
    const int grid = (int)std::min<size_t>((pixels + 255) / 256, (size_t)ctx->sm_count * 32);
    cudaEventRecord(ctx->ev0, q);
    cudaMemsetAsync(p.keys, 0xFF, 8 * pixels, q);
    cudaMemsetAsync(p.counts, 0, 4 * sizeof(unsigned long long), q);
    if (s->n_tri > 0) {
        k_raster_tris<<<(s->n_tri + 127) / 128, 128, 0, q>>>(s->dev, p, nullptr, s->n_tri);
        k_raster_big<<<ctx->sm_count * 8, 256, 0, q>>>(p);
    }
    k_raster_resolve<<<grid, 256, 0, q>>>(s->dev, p, d_bitmap, stride_bytes / 4u);
    cudaEventRecord(ctx->ev1, q);
    st = cuda_status(ctx, cudaGetLastError(), "raster kernels");
    unsigned long long counts[4] = {0, 0, 0, 0};
    if (st == MRT_OK)
        st = cuda_status(ctx, cudaMemcpyAsync(counts, p.counts, sizeof(counts), cudaMemcpyDeviceToHost, q), "raster counts");
    if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "raster preview");
    // triangles sent on by a full queue: further passes over the overflow list (only scenes whose
    // large pieces exceed the queue), the image resolved again after each
    for (int pass = 1; st == MRT_OK && counts[3] > 0; ++pass) {
        if ((uint64_t)pass > (uint64_t)s->n_tri + 1) { set_error(ctx, "mrt_raster_preview: no progress"); return MRT_ERR_LIMIT; }
        const uint32_t n_items = (uint32_t)counts[3];
        const uint32_t *in = p.overflow;
        p.overflow = in == lists[0] ? lists[1] : lists[0];
        cudaMemsetAsync(p.counts, 0, sizeof(unsigned long long), q);
        cudaMemsetAsync(p.counts + 3, 0, sizeof(unsigned long long), q);
        k_raster_tris<<<(n_items + 127) / 128, 128, 0, q>>>(s->dev, p, in, n_items);
        k_raster_big<<<ctx->sm_count * 8, 256, 0, q>>>(p);
        k_raster_resolve<<<grid, 256, 0, q>>>(s->dev, p, d_bitmap, stride_bytes / 4u);
        st = cuda_status(ctx, cudaGetLastError(), "raster kernels");
        if (st == MRT_OK)
            st = cuda_status(ctx, cudaMemcpyAsync(counts, p.counts, sizeof(counts), cudaMemcpyDeviceToHost, q), "raster counts");
        if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "raster preview");
    }
    if (st == MRT_OK && mem == MRT_MEM_HOST)
        st = cuda_status(ctx, cudaMemcpyAsync(bitmap, d_bitmap, bm_bytes, cudaMemcpyDeviceToHost, q), "bitmap out");
    if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "raster preview");
    if (st != MRT_OK) return st;
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->triangles = s->n_tri;
        stats->drawn = counts[1];
        stats->fragments = counts[2];
        stats->device_ms = ms;
    }
    return MRT_OK;
}
