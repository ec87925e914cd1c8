// mrt_trace.cuh - closest-hit and any-hit traversal on the device.
//
// Shader::rayTrace tests the accelerators in a fixed order, planes -> spheres -> triangles ->
// lights (Shader.cpp:124-150), every primitive replacing the intersection only when its distance is
// strictly below the current one (Triangle.cpp:86, Sphere.cpp:43, Plane.cpp:37).  The routines here
// keep that order and those comparisons:
//   * NAIVE, REGULAR_GRID and BVH/REFERENCE walk the reference structures in the reference order
//     with the reference box test, so the result is the reference's bit for bit;
//   * BVH/FAST walks an 8-wide tree with quantised child boxes (a Morton-ordered binary tree
//     collapsed and compressed on the device) nearest child first with a conservative box test and
//     keeps the lexicographic minimum (t, index): the Naive<T> result without visiting every triangle.
#pragma once

#include "mrt_device.cuh"

namespace mrt {

constexpr int kRefStack = 128;
constexpr uint32_t kMaxGridSteps = 1u << 20;
constexpr uint32_t kMaxBvhSteps = 1u << 24;   // traversal iterations per ray before MRT_ERR_LIMIT

MRT_HD uint32_t hid(uint32_t type, uint32_t index) { return MRT_HIT_ID(type, index); }

template <class S>
__device__ __forceinline__ void raise_error(const S &s, int code) {
    if (s.error_flag) atomicMax(s.error_flag, code);
}

// the fields of a scene the FAST-BVH node and leaf steps read; a persistent lane that traces in a
// scene of its own (batched jobs) keeps these in registers instead of re-reading its scene record
struct FastView {
    const float4 *fnodes;
    const float4 *ftris;
    uint32_t n_fnodes;
    uint32_t n_tri;
    int32_t *error_flag;
};

__device__ __forceinline__ FastView fast_view(const DevScene &s) {
    return FastView{s.fnodes, s.ftris, s.n_fnodes, s.n_tri, s.error_flag};
}

// ---------------------------------------------------------------------------------------------
// single primitives with the reference's accept rule  !(t < eps || t >= length)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool plane_hit(const DevScene &s, uint32_t i, const Ray &r, float &len, uint32_t &id) {
    const uint32_t self = hid(MRT_PRIM_PLANE, i);
    if (r.exclude == self) return false;
    float t;
    if (!pln_solve(v3(s.pln_n[i]), v3(s.pln_p[i]), r, t)) return false;
    if (t < kEpsilon || t >= len) return false;
    len = t;
    id = self;
    return true;
}
__device__ __forceinline__ bool plane_occ(const DevScene &s, uint32_t i, const Ray &r, float dist) {
    if (r.exclude == hid(MRT_PRIM_PLANE, i)) return false;
    float t;
    if (!pln_solve(v3(s.pln_n[i]), v3(s.pln_p[i]), r, t)) return false;
    return t > kEpsilon && t < dist;
}
__device__ __forceinline__ bool sphere_hit(const DevScene &s, uint32_t i, const Ray &r, float &len, uint32_t &id) {
    const float4 c = s.sph[i];
    float t;
    if (!sph_solve(v3(c), c.w, r, t)) return false;
    if (t < kSphereEpsilon || t >= len) return false;
    len = t;
    id = hid(MRT_PRIM_SPHERE, i);
    return true;
}
__device__ __forceinline__ bool sphere_occ(const DevScene &s, uint32_t i, const Ray &r, float dist) {
    const float4 c = s.sph[i];
    float t;
    if (!sph_solve(v3(c), c.w, r, t)) return false;
    return t > kSphereEpsilon && t < dist;
}
__device__ __forceinline__ bool triangle_hit(const DevScene &s, uint32_t i, const Ray &r, float &len, uint32_t &id) {
    const uint32_t self = hid(MRT_PRIM_TRIANGLE, i);
    if (r.exclude == self) return false;
    float t, u, v;
    const V3 a = v3(s.tri_a[i]), ab = v3(s.tri_ab[i]), ac = v3(s.tri_ac[i]);
    // tri_test already rejected t < Epsilon; NaN distances fall through as in the reference
    if (!tri_test(a, ab, ac, r, t, u, v)) return false;
    if (t >= len) return false;
    len = t;
    id = self;
    return true;
}
__device__ __forceinline__ bool triangle_occ(const DevScene &s, uint32_t i, const Ray &r, float dist) {
    if (r.exclude == hid(MRT_PRIM_TRIANGLE, i)) return false;
    return tri_occ(v3(s.tri_a[i]), v3(s.tri_ab[i]), v3(s.tri_ac[i]), r, dist);
}

template <int T>
__device__ __forceinline__ bool prim_hit(const DevScene &s, uint32_t i, const Ray &r, float &len, uint32_t &id) {
    if (T == kPlane) return plane_hit(s, i, r, len, id);
    if (T == kSphere) return sphere_hit(s, i, r, len, id);
    return triangle_hit(s, i, r, len, id);
}
template <int T>
__device__ __forceinline__ bool prim_occ(const DevScene &s, uint32_t i, const Ray &r, float dist) {
    if (T == kPlane) return plane_occ(s, i, r, dist);
    if (T == kSphere) return sphere_occ(s, i, r, dist);
    return triangle_occ(s, i, r, dist);
}
template <int T> __device__ __forceinline__ uint32_t prim_count(const DevScene &s) {
    return T == kPlane ? s.n_pln : (T == kSphere ? s.n_sph : s.n_tri);
}

// ---------------------------------------------------------------------------------------------
// Naive<T>::trace / shadowTrace  Naive.hpp:56-74
// ---------------------------------------------------------------------------------------------
template <int T>
__device__ bool naive_trace(const DevScene &s, const Ray &r, float &len, uint32_t &id) {
    bool hit = false;
    const uint32_t n = prim_count<T>(s);
    for (uint32_t i = 0; i < n; ++i) hit |= prim_hit<T>(s, i, r, len, id);
    return hit;
}
template <int T>
__device__ bool naive_occ(const DevScene &s, const Ray &r, float dist) {
    const uint32_t n = prim_count<T>(s);
    for (uint32_t i = 0; i < n; ++i)
        if (prim_occ<T>(s, i, r, dist)) return true;
    return false;
}

// ---------------------------------------------------------------------------------------------
// BVH<T>::trace / shadowTrace on the reference tree  BVH.hpp:158-271
// ---------------------------------------------------------------------------------------------
template <int T>
__device__ bool refbvh_trace(const DevScene &s, const Ray &r, float &len, uint32_t &id) {
    if (prim_count<T>(s) == 0) return false;
    const RefNode *nodes = s.rnodes[T];
    uint32_t stack[kRefStack];
    int sp = 1;
    stack[0] = 0;
    uint32_t node = 0;
    bool hit = false;
    uint32_t steps = 0;
    const uint32_t n_nodes = s.rnode_count[T];
    do {
        if (node >= n_nodes || ++steps > kMaxBvhSteps) { raise_error(s, MRT_ERR_LIMIT); return hit; }
        const RefNode nd = nodes[node];
        if (ref_box_hit(nd.mn, nd.mx, r)) {
            if (nd.count > 0) {
                if (nd.offset + nd.count > prim_count<T>(s)) { raise_error(s, MRT_ERR_LIMIT); return hit; }
                for (uint32_t i = 0; i < nd.count; ++i) hit |= prim_hit<T>(s, nd.offset + i, r, len, id);
                --sp;
                node = stack[sp];
            } else {
                const uint32_t left = nd.offset, right = left + 1;
                if (right >= n_nodes) { raise_error(s, MRT_ERR_LIMIT); return hit; }
                const bool tl = ref_box_hit(nodes[left].mn, nodes[left].mx, r);
                const bool tr = ref_box_hit(nodes[right].mn, nodes[right].mx, r);
                if (!tl && !tr) {
                    --sp;
                    node = stack[sp];
                } else {
                    node = tl ? left : right;
                    if (tl && tr) {
                        if (sp >= kRefStack) { raise_error(s, MRT_ERR_LIMIT); return hit; }
                        stack[sp++] = right;
                    }
                }
            }
        } else {
            --sp;
            node = stack[sp];
        }
    } while (sp > 0);
    return hit;
}

template <int T>
__device__ bool refbvh_occ(const DevScene &s, const Ray &r, float dist) {
    if (prim_count<T>(s) == 0) return false;
    const RefNode *nodes = s.rnodes[T];
    uint32_t stack[kRefStack];
    int sp = 1;
    stack[0] = 0;
    uint32_t node = 0;
    uint32_t steps = 0;
    const uint32_t n_nodes = s.rnode_count[T];
    do {
        if (node >= n_nodes || ++steps > kMaxBvhSteps) { raise_error(s, MRT_ERR_LIMIT); return false; }
        const RefNode nd = nodes[node];
        if (ref_box_hit(nd.mn, nd.mx, r)) {
            if (nd.count > 0) {
                if (nd.offset + nd.count > prim_count<T>(s)) { raise_error(s, MRT_ERR_LIMIT); return false; }
                for (uint32_t i = 0; i < nd.count; ++i)
                    if (prim_occ<T>(s, nd.offset + i, r, dist)) return true;
                --sp;
                node = stack[sp];
            } else {
                const uint32_t left = nd.offset, right = left + 1;
                if (right >= n_nodes) { raise_error(s, MRT_ERR_LIMIT); return false; }
                const bool tl = ref_box_hit(nodes[left].mn, nodes[left].mx, r);
                const bool tr = ref_box_hit(nodes[right].mn, nodes[right].mx, r);
                if (!tl && !tr) {
                    --sp;
                    node = stack[sp];
                } else {
                    node = tl ? left : right;
                    if (tl && tr) {
                        if (sp >= kRefStack) { raise_error(s, MRT_ERR_LIMIT); return false; }
                        stack[sp++] = right;
                    }
                }
            }
        } else {
            --sp;
            node = stack[sp];
        }
    } while (sp > 0);
    return false;
}

// ---------------------------------------------------------------------------------------------
// RegularGrid<T>::trace / shadowTrace  RegularGrid.hpp:157-465
// ---------------------------------------------------------------------------------------------
struct Dda {
    int32_t X, Y, Z;
    int32_t sx, sy, sz, ox, oy, oz;
    float tx, ty, tz, dx, dy, dz;
};

__device__ __forceinline__ uint32_t grid_cell(const DevGrid &g, int32_t X, int32_t Y, int32_t Z) {
    if (g.index_mode == MRT_GRID_INDEX_LINEAR)
        return (uint32_t)X + (uint32_t)Y * (uint32_t)g.G + (uint32_t)Z * (uint32_t)g.G * (uint32_t)g.G;
    return (uint32_t)X + ((uint32_t)Y << g.shift) + ((uint32_t)Z << (g.shift * 2u));
}

// DDA setup, RegularGrid.hpp:161-231
__device__ __forceinline__ void dda_setup(const DevGrid &g, const Ray &r, Dda &s) {
    const V3 cell = (r.o - g.mn) * g.sr;
    int32_t X = f2i_x86(cell.x), Y = f2i_x86(cell.y), Z = f2i_x86(cell.z);
    X = X > 0 ? X : 0; Y = Y > 0 ? Y : 0; Z = Z > 0 ? Z : 0;
    X = (g.G - 1 < X) ? g.G - 1 : X; Y = (g.G - 1 < Y) ? g.G - 1 : Y; Z = (g.G - 1 < Z) ? g.G - 1 : Z;
    float cbx, cby, cbz;
    if (r.d.x > 0) { s.sx = 1; s.ox = g.G; cbx = g.mn.x + (float)(X + 1) * g.cw.x; }
    else { s.sx = -1; s.ox = -1; cbx = g.mn.x + (float)X * g.cw.x; }
    if (r.d.y > 0) { s.sy = 1; s.oy = g.G; cby = g.mn.y + (float)(Y + 1) * g.cw.y; }
    else { s.sy = -1; s.oy = -1; cby = g.mn.y + (float)Y * g.cw.y; }
    if (r.d.z > 0) { s.sz = 1; s.oz = g.G; cbz = g.mn.z + (float)(Z + 1) * g.cw.z; }
    else { s.sz = -1; s.oz = -1; cbz = g.mn.z + (float)Z * g.cw.z; }
    s.dx = s.dy = s.dz = 0.0f;
    if (fabsf(r.d.x) > kEpsilon) { const float rr = 1.0f / r.d.x; s.tx = (cbx - r.o.x) * rr; s.dx = g.cw.x * (float)s.sx * rr; }
    else s.tx = kRayLengthMax;
    if (fabsf(r.d.y) > kEpsilon) { const float rr = 1.0f / r.d.y; s.ty = (cby - r.o.y) * rr; s.dy = g.cw.y * (float)s.sy * rr; }
    else s.ty = kRayLengthMax;
    if (fabsf(r.d.z) > kEpsilon) { const float rr = 1.0f / r.d.z; s.tz = (cbz - r.o.z) * rr; s.dz = g.cw.z * (float)s.sz * rr; }
    else s.tz = kRayLengthMax;
    s.X = X; s.Y = Y; s.Z = Z;
}

// one step of the first walk; false when the walk leaves the grid (RegularGrid.hpp:251-279)
__device__ __forceinline__ bool dda_step(Dda &s) {
    if (s.tx < s.ty) {
        if (s.tx < s.tz) { s.X += s.sx; if (s.X == s.ox) return false; s.tx = s.tx + s.dx; }
        else { s.Z += s.sz; if (s.Z == s.oz) return false; s.tz = s.tz + s.dz; }
    } else {
        if (s.ty < s.tz) { s.Y += s.sy; if (s.Y == s.oy) return false; s.ty = s.ty + s.dy; }
        else { s.Z += s.sz; if (s.Z == s.oz) return false; s.tz = s.tz + s.dz; }
    }
    return true;
}

// cells visited (start[c], start[c + 1] read) and references tested (refs[k] and the primitive read)
struct GridCounts {
    uint32_t cells;
    uint32_t refs;
};

template <int T, bool kCount = false>
__device__ bool grid_trace(const DevScene &s, const Ray &r, float &len, uint32_t &id, GridCounts *cnt = nullptr) {
    const DevGrid &g = s.grid[T];
    if (!g.has) return false;
    Dda st;
    dda_setup(g, r, st);
    bool hit = false;
    uint32_t steps = 0;
    for (;;) {
        const uint32_t c = grid_cell(g, st.X, st.Y, st.Z);
        const uint32_t b = g.start[c], e = g.start[c + 1];
        if (kCount) cnt->cells++;
        bool found = false;
        for (uint32_t k = b; k < e; ++k) {
            if (kCount) cnt->refs++;
            hit |= prim_hit<T>(s, g.refs[k], r, len, id);
            if (hit) { found = true; break; }
        }
        if (found) break;
        if (!dda_step(st)) return hit;
        if (++steps > kMaxGridSteps) { raise_error(s, MRT_ERR_LIMIT); return hit; }
    }
    for (;;) {   // testloop, RegularGrid.hpp:282-335
        const uint32_t c = grid_cell(g, st.X, st.Y, st.Z);
        const uint32_t b = g.start[c], e = g.start[c + 1];
        if (kCount) { cnt->cells++; cnt->refs += e - b; }
        for (uint32_t k = b; k < e; ++k) hit |= prim_hit<T>(s, g.refs[k], r, len, id);
        if (st.tx < st.ty) {
            if (st.tx < st.tz) {
                if (len < st.tx) break;
                st.X += st.sx; if (st.X == st.ox) break; st.tx = st.tx + st.dx;
            } else {
                if (len < st.tz) break;
                st.Z += st.sz; if (st.Z == st.oz) break; st.tz = st.tz + st.dz;
            }
        } else {
            if (st.ty < st.tz) {
                if (len < st.ty) break;
                st.Y += st.sy; if (st.Y == st.oy) break; st.ty = st.ty + st.dy;
            } else {
                if (len < st.tz) break;
                st.Z += st.sz; if (st.Z == st.oz) break; st.tz = st.tz + st.dz;
            }
        }
        if (++steps > kMaxGridSteps) { raise_error(s, MRT_ERR_LIMIT); break; }
    }
    return hit;
}

template <int T>
__device__ bool grid_occ(const DevScene &s, const Ray &r, float dist) {
    const DevGrid &g = s.grid[T];
    if (!g.has) return false;
    Dda st;
    dda_setup(g, r, st);
    uint32_t steps = 0;
    for (;;) {
        const uint32_t c = grid_cell(g, st.X, st.Y, st.Z);
        const uint32_t b = g.start[c], e = g.start[c + 1];
        for (uint32_t k = b; k < e; ++k)
            if (prim_occ<T>(s, g.refs[k], r, dist)) return true;
        if (!dda_step(st)) return false;
        if (++steps > kMaxGridSteps) { raise_error(s, MRT_ERR_LIMIT); return false; }
    }
}

// ---------------------------------------------------------------------------------------------
// FAST BVH: 8-wide nodes of 128 bytes with 16-bit quantised child boxes, one node per traversal
// step.  A node's internal children are stored contiguously from its child base (in slot order), the
// triangles of its leaf children contiguously from its triangle base (48-byte records A|index, AB,
// AC).  The compressed wide node and its traversal by node groups (a base index and a bit mask of the
// children still to visit, one stack entry per node instead of one per child) follow Ylitie, Karras
// and Laine, "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs" (HPG 2017);
// here the boxes are quantised to 16 bits and every plane distance is bounded by directed rounding.
//
// Node, 32 words (the fnodes array holds n_fnodes of them), in two 64-byte halves that each hold what
// the test of four children reads (word positions: kNodeChildBase, kNodeTriBase, kNodeMeta and
// node_plane_word() in mrt_device.cuh):
//   w[0..2]  origin p of the quantisation grid (floats)
//   w[3]     ex | ey << 8 | ez << 16 (axis a's grid step is 2^(e_a - 127)) | imask << 24 (slots
//            holding internal children)
//   w[4..15] slots 0-3's box on x (w[4..7]), y (w[8..11]), z (w[12..15]): qlo | qhi << 16, the planes
//            p + step * q; the quantised box contains the exact box of everything below the slot
//   w[16]    child base: node index of the first internal child
//   w[17]    triangle base: record index of the first triangle of the leaf children
//   w[18..19] one byte per slot: a leaf child's triangle bits (1, 3 or 7 for 1..3 triangles) << 5 | the
//            offset of its first triangle from the triangle base; 0 for internal and empty slots
//   w[20..31] slots 4-7's box on x, y, z as w[4..15]
// Slots are assigned by the octant of the child's centre within the node, so visiting the children
// in the order slot ^ octant(ray direction) is close to front to back.
// ---------------------------------------------------------------------------------------------

// A ray prepared for the quantised box test: 1/d (components of |d| < 1e-20 replaced by +-1e-20) and
// the octant of the direction.  With A = step * (1/d) (exact: a power of two times a float) the
// distance of plane p + step * q is (p - o) / d + q * A; the entry distance is computed rounded down
// from a lower bound of (p - o) / d (built from o * (1/d) rounded up), the exit distance rounded up
// from an upper bound, so with respect to the rounded 1/d the test never rejects a box the ray
// touches.  The rounding of 1/d itself is relative and covered by the 1e-6 tolerance of the
// comparison.  The grid offset q enters as the float 2^23 + q (built by one byte permute) with
// 2^23 * A folded into the bound, which loosens a plane by at most one grid step (1/65535 of the
// node's extent).
struct FastRay {
    V3 inv;
    uint32_t oct;    // bit a: the direction is negative along axis a
};

__device__ __forceinline__ FastRay fast_ray(const Ray &r) {
    FastRay f;
    const float e = 1e-20f;
    const float dx = fabsf(r.d.x) < e ? copysignf(e, r.d.x) : r.d.x;
    const float dy = fabsf(r.d.y) < e ? copysignf(e, r.d.y) : r.d.y;
    const float dz = fabsf(r.d.z) < e ? copysignf(e, r.d.z) : r.d.z;
    f.inv = V3{1.0f / dx, 1.0f / dy, 1.0f / dz};
    f.oct = (f.inv.x < 0.0f ? 1u : 0u) | (f.inv.y < 0.0f ? 2u : 0u) | (f.inv.z < 0.0f ? 4u : 0u);
    return f;
}

struct FastCounts {
    uint32_t nodes;  // 128-byte nodes fetched
    uint32_t tris;   // 48-byte triangle records fetched
};

// the children of one node that the ray segment [0, tmax] may touch
struct NodeHits {
    uint32_t child_base;   // node index of the node's first internal child
    uint32_t groups;       // imask << 8 | internal children hit, bit (slot ^ ray octant)
    uint32_t tri_base;     // record index of the node's first leaf triangle
    uint32_t tris;         // leaf triangles hit: bit j is record tri_base + j
};

__device__ __forceinline__ uint32_t uint4_word(const uint4 &a, int k) {
    switch (k & 3) {
        case 0: return a.x; case 1: return a.y; case 2: return a.z; default: return a.w;
    }
}

// 2^23 + (lo or hi half of w) as a float: byte permute of w with 0x4B000000 (selector 0x7410 takes
// the low half, 0x7432 the high half)
__device__ __forceinline__ float grid_offset(uint32_t w, uint32_t sel) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, sel));
}

// three-input minimum and maximum (one instruction each on sm_100; NaN inputs are ignored as by
// fminf / fmaxf)
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// bit s of an 8-bit slot mask moved to bit s ^ oct (the visiting key of slot s)
__device__ __forceinline__ uint32_t slots_to_keys(uint32_t m, uint32_t oct) {
    if (oct & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
    if (oct & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
    if (oct & 4u) m = ((m & 0x0Fu) << 4) | ((m >> 4) & 0x0Fu);
    return m;
}

// 32 bytes at a 32-byte-aligned address as one load (sm_100: 256-bit loads), through the read-only path
#ifndef MRT_NODE_LDG256
#define MRT_NODE_LDG256 1
#endif
__device__ __forceinline__ void ldg_32b(const uint4 *p, uint4 &a, uint4 &b) {
#if MRT_NODE_LDG256
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
        : "l"(p));
#else
    a = __ldg(p);
    b = __ldg(p + 1);
#endif
}

// the four children of one half-node (planes x, y, z of slots 4h..4h+3) against the ray: bit k of the
// result is slot 4h + k's box possibly touched
__device__ __forceinline__ uint32_t half_hits(const uint4 &xq, const uint4 &yq, const uint4 &zq, float ax, float ay,
                                              float az, float lox, float loy, float loz, float hix, float hiy,
                                              float hiz, uint32_t nx, uint32_t ny, uint32_t nz, float tmax) {
    uint32_t hits = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t wx = uint4_word(xq, j), wy = uint4_word(yq, j), wz = uint4_word(zq, j);
        const float tnx = __fmaf_rd(grid_offset(wx, nx), ax, lox), tfx = __fmaf_ru(grid_offset(wx, nx ^ 0x22u), ax, hix);
        const float tny = __fmaf_rd(grid_offset(wy, ny), ay, loy), tfy = __fmaf_ru(grid_offset(wy, ny ^ 0x22u), ay, hiy);
        const float tnz = __fmaf_rd(grid_offset(wz, nz), az, loz), tfz = __fmaf_ru(grid_offset(wz, nz ^ 0x22u), az, hiz);
        const float tn = max3f(tnx, tny, fmaxf(tnz, 0.0f));
        const float tf = min3f(tfx, tfy, fminf(tfz, tmax));
        if (tn <= tf * 1.000001f) hits |= 1u << j;
    }
    return hits;
}

template <class S>
__device__ __forceinline__ NodeHits node_hits(const S &s, uint32_t node, const FastRay &f, const V3 &o, float tmax) {
    const uint4 *p = reinterpret_cast<const uint4 *>(s.fnodes) + (size_t)node * (kNodeWords / 4);
    // first half: grid origin, exponents and internal mask; planes of slots 0-3 on x, y, z
    uint4 h0, x0, y0, z0;
    ldg_32b(p, h0, x0);
    ldg_32b(p + 2, y0, z0);
    // per axis: A = step / d, and bounds of (p - o) / d - 2^23 A
    const float ax = __uint_as_float((h0.w & 0xFFu) << 23) * f.inv.x;
    const float ay = __uint_as_float(((h0.w >> 8) & 0xFFu) << 23) * f.inv.y;
    const float az = __uint_as_float(((h0.w >> 16) & 0xFFu) << 23) * f.inv.z;
    const float lox = __fmaf_rd(-8388608.0f, ax, __fmaf_rd(__uint_as_float(h0.x), f.inv.x, -__fmul_ru(o.x, f.inv.x)));
    const float loy = __fmaf_rd(-8388608.0f, ay, __fmaf_rd(__uint_as_float(h0.y), f.inv.y, -__fmul_ru(o.y, f.inv.y)));
    const float loz = __fmaf_rd(-8388608.0f, az, __fmaf_rd(__uint_as_float(h0.z), f.inv.z, -__fmul_ru(o.z, f.inv.z)));
    const float hix = __fmaf_ru(-8388608.0f, ax, __fmaf_ru(__uint_as_float(h0.x), f.inv.x, -__fmul_rd(o.x, f.inv.x)));
    const float hiy = __fmaf_ru(-8388608.0f, ay, __fmaf_ru(__uint_as_float(h0.y), f.inv.y, -__fmul_rd(o.y, f.inv.y)));
    const float hiz = __fmaf_ru(-8388608.0f, az, __fmaf_ru(__uint_as_float(h0.z), f.inv.z, -__fmul_rd(o.z, f.inv.z)));
    // the entry plane is the lo plane where the direction is positive
    const uint32_t nx = 0x7410u + ((f.oct & 1u) ? 0x22u : 0u);
    const uint32_t ny = 0x7410u + ((f.oct & 2u) ? 0x22u : 0u);
    const uint32_t nz = 0x7410u + ((f.oct & 4u) ? 0x22u : 0u);
    const uint32_t imask = h0.w >> 24;
    uint32_t hits = half_hits(x0, y0, z0, ax, ay, az, lox, loy, loz, hix, hiy, hiz, nx, ny, nz, tmax);
    // second half: child base, triangle base, leaf meta bytes; planes of slots 4-7
    uint4 h1, x1, y1, z1;
    ldg_32b(p + 4, h1, x1);
    ldg_32b(p + 6, y1, z1);
    hits |= half_hits(x1, y1, z1, ax, ay, az, lox, loy, loz, hix, hiy, hiz, nx, ny, nz, tmax) << 4;
    // the triangles of the leaf children hit (meta byte k: triangle bits << 5 | offset)
    uint32_t tris = 0;
    for (uint32_t lh = hits & ~imask; lh; lh &= lh - 1u) {
        const uint32_t meta = __byte_perm(h1.z, h1.w, (uint32_t)(__ffs(lh) - 1)) & 0xFFu;
        tris |= (meta >> 5) << (meta & 31u);
    }
    return NodeHits{h1.x, (imask << 8) | slots_to_keys(hits & imask, f.oct), h1.y, tris};
}

// node index of the child at visiting key `key` of a group (child base, imask << 8 | ...)
__device__ __forceinline__ uint32_t group_node(uint32_t base, uint32_t groups, uint32_t key, uint32_t oct) {
    const uint32_t slot = key ^ oct;
    return base + __popc((groups >> 8) & ((1u << slot) - 1u));
}

template <bool kCount, class S>
__device__ __forceinline__ void fast_tris(const S &s, const Ray &r, uint32_t base, uint32_t bits, float &best_t,
                                          uint32_t &best_id, FastCounts &cnt) {
    while (bits) {
        const uint32_t k = base + (uint32_t)(__ffs(bits) - 1);
        bits &= bits - 1u;
        if (k >= s.n_tri) { raise_error(s, MRT_ERR_LIMIT); return; }
        const float4 A = __ldg(&s.ftris[3 * (size_t)k]);
        const float4 AB = __ldg(&s.ftris[3 * (size_t)k + 1]);
        const float4 AC = __ldg(&s.ftris[3 * (size_t)k + 2]);
        if (kCount) cnt.tris++;
        const uint32_t id = hid(MRT_PRIM_TRIANGLE, __float_as_uint(A.w));
        if (r.exclude == id) continue;
        float t, u, v;
        if (!tri_test(v3(A), v3(AB), v3(AC), r, t, u, v)) continue;
        // a tie goes to the lower triangle index; a plane or sphere found first (smaller ids) and
        // the incoming length with no hit (MRT_HIT_NONE) keep a tie, as the reference's strict `<`
        if (t < best_t || (t == best_t && id < best_id && best_id != MRT_HIT_NONE)) {
            best_t = t;
            best_id = id;
        }
    }
}

template <class S>
__device__ __forceinline__ bool fast_tris_occ(const S &s, const Ray &r, uint32_t base, uint32_t bits, float dist) {
    while (bits) {
        const uint32_t k = base + (uint32_t)(__ffs(bits) - 1);
        bits &= bits - 1u;
        if (k >= s.n_tri) { raise_error(s, MRT_ERR_LIMIT); return false; }
        const float4 A = __ldg(&s.ftris[3 * (size_t)k]);
        const float4 AB = __ldg(&s.ftris[3 * (size_t)k + 1]);
        const float4 AC = __ldg(&s.ftris[3 * (size_t)k + 2]);
        if (r.exclude == hid(MRT_PRIM_TRIANGLE, __float_as_uint(A.w))) continue;
        if (tri_occ(v3(A), v3(AB), v3(AC), r, dist)) return true;
    }
    return false;
}

// ---------------------------------------------------------------------------------------------
// resumable traversal state of one ray (closest hit; any hit keeps best_t = the shadow distance and
// sets `have` at the first occluder).  The stack holds node groups, at most one per tree level.
// ---------------------------------------------------------------------------------------------
constexpr int kFastStack = 64;   // the tree is at most 62 levels deep (30-bit Morton codes + 32 index bits)

struct FastTrav {
    FastRay f;
    float best_t;      // closest hit so far (any hit: the shadow distance)
    uint32_t best_id;  // its hit id: the plane or sphere hit before the tree, MRT_HIT_NONE, or a
                       // triangle (for an any-hit query: a triangle id once occluded)
    uint32_t g_base, g_bits;     // node group being expanded: child base, imask << 8 | keys left
    uint32_t t_base, t_bits;     // triangles waiting for the leaf phase
    uint32_t t2_base, t2_bits;   // a second group of them, found while the warp still searched
    int sp;
    uint32_t c_nodes, c_tris;
};

// the tree answered: a triangle is the closest hit (any hit: an occluder was found)
__device__ __forceinline__ bool trav_hit(const FastTrav &t) { return MRT_HIT_TYPE(t.best_id) == MRT_PRIM_TRIANGLE; }
__device__ __forceinline__ void trav_set_occluded(FastTrav &t) { t.best_id = hid(MRT_PRIM_TRIANGLE, 0u); }

// the stack of node groups in local memory
struct TravStack {
    uint2 e[kFastStack];
    __device__ __forceinline__ void put(int i, uint2 v) { e[i] = v; }
    __device__ __forceinline__ uint2 get(int i) const { return e[i]; }
};

template <bool kCount, class S>
__device__ __forceinline__ void trav_begin(const S &s, const Ray &r, float len0, uint32_t id0, FastTrav &t) {
    t.f = fast_ray(r);
    t.best_t = len0;
    t.best_id = id0;
    t.g_base = 0;
    // the root as the only internal child (slot 0) of a virtual group
    t.g_bits = s.n_tri == 0 ? 0u : ((1u << 8) | (1u << t.f.oct));
    t.t_bits = 0;
    t.t2_bits = 0;
    t.sp = 0;
    t.c_nodes = 0;
    t.c_tris = 0;
}

__device__ __forceinline__ bool trav_has_nodes(const FastTrav &t) { return (t.g_bits & 0xFFu) != 0u || t.sp > 0; }
__device__ __forceinline__ bool trav_has_leaf(const FastTrav &t) { return t.t_bits != 0u; }
__device__ __forceinline__ bool trav_wants_node(const FastTrav &t) { return t.t_bits == 0u && trav_has_nodes(t); }
// a lane with triangles waiting may go on with node steps while others of its warp still search
// (Aila and Laine, "Understanding the efficiency of ray traversal on GPUs", HPG 2009: speculative
// traversal), up to a second group of triangles
__device__ __forceinline__ bool trav_can_speculate(const FastTrav &t) {
    return t.t_bits != 0u && t.t2_bits == 0u && trav_has_nodes(t);
}
__device__ __forceinline__ bool trav_finished(const FastTrav &t) {
    return t.t_bits == 0u && t.t2_bits == 0u && !trav_has_nodes(t);
}
// nothing left to do (an error, or the first occluder of an any-hit query)
__device__ __forceinline__ void trav_clear(FastTrav &t) {
    t.g_bits = 0;
    t.sp = 0;
    t.t_bits = 0;
    t.t2_bits = 0;
}

template <class S>
__device__ __forceinline__ bool node_in_range(const S &s, uint32_t node) {
    return node < s.n_fnodes;
}

// one node step: the next child of the current group (a group popped first when it is empty), its
// node tested, its hit internal children becoming the current group (the rest of the old one pushed)
template <bool kCount, class S, class Stack>
__device__ __forceinline__ void trav_node_step(const S &s, const Ray &r, FastTrav &t, Stack &st) {
    if ((t.g_bits & 0xFFu) == 0u) {
        if (t.sp == 0) return;
        const uint2 e = st.get(--t.sp);
        t.g_base = e.x;
        t.g_bits = e.y;
    }
    const uint32_t key = (uint32_t)(__ffs(t.g_bits & 0xFFu) - 1);
    t.g_bits &= ~(1u << key);
    const uint32_t node = group_node(t.g_base, t.g_bits, key, t.f.oct);
    if (t.g_bits & 0xFFu) {
        if (t.sp >= kFastStack) { raise_error(s, MRT_ERR_LIMIT); trav_clear(t); return; }
        st.put(t.sp++, make_uint2(t.g_base, t.g_bits));
    }
    if (!node_in_range(s, node)) { raise_error(s, MRT_ERR_LIMIT); trav_clear(t); return; }
    const NodeHits h = node_hits(s, node, t.f, r.o, t.best_t);
    if (kCount) t.c_nodes++;
    t.g_base = h.child_base;
    t.g_bits = h.groups;
    if (h.tris) {
        if (t.t_bits == 0u) { t.t_base = h.tri_base; t.t_bits = h.tris; }
        else { t.t2_base = h.tri_base; t.t2_bits = h.tris; }
    }
}

template <bool kCount, class S>
__device__ __forceinline__ void trav_leaf_step(const S &s, const Ray &r, FastTrav &t) {
    FastCounts cnt{0, 0};
    fast_tris<kCount>(s, r, t.t_base, t.t_bits, t.best_t, t.best_id, cnt);
    if (t.t2_bits) fast_tris<kCount>(s, r, t.t2_base, t.t2_bits, t.best_t, t.best_id, cnt);
    if (kCount) t.c_tris += cnt.tris;
    t.t_bits = 0;
    t.t2_bits = 0;
}

// any-hit leaf step on the same state (best_t holds the shadow distance): the first occluder ends
// the query with `have` set
template <class S>
__device__ __forceinline__ void trav_occ_leaf_step(const S &s, const Ray &r, FastTrav &t) {
    if (fast_tris_occ(s, r, t.t_base, t.t_bits, t.best_t) ||
        (t.t2_bits && fast_tris_occ(s, r, t.t2_base, t.t2_bits, t.best_t))) {
        trav_set_occluded(t);
        trav_clear(t);
        return;
    }
    t.t_bits = 0;
    t.t2_bits = 0;
}

// closest triangle with the reference's accept rule against the incoming length `len` (one ray per
// thread): lexicographic minimum (t, index) over the triangles of every box the ray may touch
template <bool kCount = false>
__device__ bool fast_trace(const DevScene &s, const Ray &r, float &len, uint32_t &id, FastCounts *counts = nullptr) {
    if (s.n_tri == 0) return false;
    FastTrav t;
    TravStack st;
    trav_begin<kCount>(s, r, len, id, t);
    uint32_t steps = 0;
    while (!trav_finished(t)) {
        if (trav_has_leaf(t)) {
            trav_leaf_step<kCount>(s, r, t);
        } else {
            if (++steps > kMaxBvhSteps) { raise_error(s, MRT_ERR_LIMIT); break; }
            trav_node_step<kCount>(s, r, t, st);
        }
    }
    if (counts) *counts = FastCounts{t.c_nodes, t.c_tris};
    if (!trav_hit(t)) return false;
    len = t.best_t;
    id = t.best_id;
    return true;
}

__device__ inline bool fast_occ(const DevScene &s, const Ray &r, float dist) {
    if (s.n_tri == 0) return false;
    FastTrav t;
    TravStack st;
    trav_begin<false>(s, r, dist, MRT_HIT_NONE, t);
    uint32_t steps = 0;
    while (!trav_finished(t)) {
        if (trav_has_leaf(t)) {
            trav_occ_leaf_step(s, r, t);
        } else {
            if (++steps > kMaxBvhSteps) { raise_error(s, MRT_ERR_LIMIT); return false; }
            trav_node_step<false>(s, r, t, st);
        }
    }
    return trav_hit(t);
}

// ---------------------------------------------------------------------------------------------
// scene-level closest hit / any hit (Shader::rayTrace / shadowTrace accelerator part)
// ---------------------------------------------------------------------------------------------
template <int ACCEL, int MODE, int T>
__device__ __forceinline__ bool trace_type(const DevScene &s, const Ray &r, float &len, uint32_t &id) {
    if (ACCEL == MRT_ACCEL_NAIVE) return naive_trace<T>(s, r, len, id);
    if (ACCEL == MRT_ACCEL_REGULAR_GRID) return grid_trace<T>(s, r, len, id);
    if (MODE == MRT_BVH_REFERENCE) return refbvh_trace<T>(s, r, len, id);
    // BVH/FAST: planes and spheres are few and walked in order; triangles use the fast tree
    if (T == kTriangle) return fast_trace<false>(s, r, len, id);
    return naive_trace<T>(s, r, len, id);
}

template <int ACCEL, int MODE, int T>
__device__ __forceinline__ bool occ_type(const DevScene &s, const Ray &r, float dist) {
    if (ACCEL == MRT_ACCEL_NAIVE) return naive_occ<T>(s, r, dist);
    if (ACCEL == MRT_ACCEL_REGULAR_GRID) return grid_occ<T>(s, r, dist);
    if (MODE == MRT_BVH_REFERENCE) return refbvh_occ<T>(s, r, dist);
    if (T == kTriangle) return fast_occ(s, r, dist);
    return naive_occ<T>(s, r, dist);
}

// Scene::traceLights, Scene.cpp:31-37 (point lights are never hit, PointLight.cpp:24-26)
__device__ __forceinline__ bool lights_trace(const DevScene &s, const Ray &r, float &len, uint32_t &id) {
    bool hit = false;
    for (uint32_t k = 0; k < s.n_light; ++k) {
        const DevLight &l = s.lights[k];
        if (l.kind != MRT_LIGHT_AREA) continue;
        float t, u, v;
        if (!tri_test(l.a, l.ab, l.ac, r, t, u, v)) continue;
        if (t >= len) continue;
        len = t;
        id = hid(MRT_PRIM_LIGHT, k);
        hit = true;
    }
    return hit;
}

template <int ACCEL, int MODE>
__device__ __forceinline__ bool scene_closest(const DevScene &s, const Ray &r, float &len, uint32_t &id) {
    len = kRayLengthMax;
    id = MRT_HIT_NONE;
    bool hit = false;
    hit |= trace_type<ACCEL, MODE, kPlane>(s, r, len, id);
    hit |= trace_type<ACCEL, MODE, kSphere>(s, r, len, id);
    hit |= trace_type<ACCEL, MODE, kTriangle>(s, r, len, id);
    hit |= lights_trace(s, r, len, id);
    return hit;
}

template <int ACCEL, int MODE>
__device__ __forceinline__ bool scene_occ(const DevScene &s, const Ray &r, float dist) {
    bool occ = false;
    occ |= occ_type<ACCEL, MODE, kPlane>(s, r, dist);
    occ |= occ_type<ACCEL, MODE, kSphere>(s, r, dist);
    occ |= occ_type<ACCEL, MODE, kTriangle>(s, r, dist);
    return occ;
}

// ---------------------------------------------------------------------------------------------
// the Intersection record of the accepted primitive (recomputed from the hit id; the values do
// not depend on the incoming length, so they equal the ones the accepting test produced)
// ---------------------------------------------------------------------------------------------
struct Isect {
    V3 point, normal, color;
    float length;
    int32_t mat;        // materialId_
    int32_t light;      // >= 0: hit an area light, material = its radiance
    uint32_t prim;      // primitive_ as a hit id (spheres: none)
};

__device__ __forceinline__ bool make_isect(const DevScene &s, const Ray &r, uint32_t id, Isect &it) {
    const uint32_t type = MRT_HIT_TYPE(id), i = MRT_HIT_INDEX(id);
    it.light = -1;
    it.color = V3{1.0f, 1.0f, 1.0f};   // Intersection.hpp:29 default primitiveColor
    if (type == MRT_PRIM_TRIANGLE || type == MRT_PRIM_LIGHT) {
        V3 a, ab, ac;
        if (type == MRT_PRIM_TRIANGLE) { a = v3(s.tri_a[i]); ab = v3(s.tri_ab[i]); ac = v3(s.tri_ac[i]); }
        else { const DevLight &l = s.lights[i]; a = l.a; ab = l.ab; ac = l.ac; }
        float t, u, v;
        if (!tri_test(a, ab, ac, r, t, u, v)) return false;
        const float w = 1.0f - u - v;   // Triangle.cpp:92-97
        if (type == MRT_PRIM_TRIANGLE) {
            const float *n = s.tri_n + 9 * (size_t)i;
            const float *c = s.tri_c + 9 * (size_t)i;
            it.normal = (V3{n[0], n[1], n[2]} * w + V3{n[3], n[4], n[5]} * u) + V3{n[6], n[7], n[8]} * v;
            it.color = (V3{c[0], c[1], c[2]} * w + V3{c[3], c[4], c[5]} * u) + V3{c[6], c[7], c[8]} * v;
            it.mat = s.tri_mat[i];
        } else {
            const V3 n = s.lights[i].na;
            it.normal = (n * w + n * u) + n * v;
            it.color = V3{0.0f, 0.0f, 0.0f};
            it.mat = -1;
            it.light = (int32_t)i;
        }
        it.point = r.o + r.d * t;
        it.length = t;
        it.prim = id;
        return true;
    }
    if (type == MRT_PRIM_SPHERE) {   // Sphere.cpp:45-50
        const float4 c = s.sph[i];
        float t;
        if (!sph_solve(v3(c), c.w, r, t)) return false;
        it.point = r.o + r.d * t;
        it.normal = normalize(it.point - v3(c));
        it.length = t;
        it.mat = s.sph_mat[i];
        it.prim = MRT_HIT_NONE;
        return true;
    }
    float t;   // plane, Plane.cpp:39-44
    if (!pln_solve(v3(s.pln_n[i]), v3(s.pln_p[i]), r, t)) return false;
    it.point = r.o + r.d * t;
    it.normal = v3(s.pln_n[i]);
    it.length = t;
    it.mat = s.pln_mat[i];
    it.prim = id;
    return true;
}

}  // namespace mrt
