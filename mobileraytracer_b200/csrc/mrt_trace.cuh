// mrt_trace.cuh - closest-hit and any-hit traversal on the device.
//
// Shader::rayTrace tests the accelerators in a fixed order, planes -> spheres -> triangles ->
// lights (Shader.cpp:124-150), every primitive replacing the intersection only when its distance is
// strictly below the current one (Triangle.cpp:86, Sphere.cpp:43, Plane.cpp:37).  The routines here
// keep that order and those comparisons:
//   * NAIVE, REGULAR_GRID and BVH/REFERENCE walk the reference structures in the reference order
//     with the reference box test, so the result is the reference's bit for bit;
//   * BVH/FAST walks a 4-wide tree (a Morton-ordered binary tree collapsed on the device) front to
//     back with a conservative box test and keeps the lexicographic minimum (t, index): the
//     Naive<T> result without visiting every triangle.
#pragma once

#include "mrt_device.cuh"

namespace mrt {

constexpr int kFastStack = 128;           // entries of the FAST traversal stack (3 pushes per node at most)
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
// FAST BVH: Morton-ordered binary tree, child pairs adjacent (64 B per pair), triangles in leaf
// order as 48-byte records.  Conservative slab test against padded boxes; front-to-back order
// with the entry distance kept on the stack.
// ---------------------------------------------------------------------------------------------
// A ray prepared for the conservative box test of the FAST tree.  The plane distances are computed
// as fma(plane, inv, -c) with c = o * inv moved outward by a margin (2^-20 |o * inv|, more than the
// rounding of o * inv and of the shift itself), so the entry distance is never overestimated and the
// exit distance never underestimated; the remaining rounding is relative and covered by the 1e-6
// tolerance of the comparison.  The test may therefore accept a box the ray misses, never reject one
// it touches.
struct FastRay {
    V3 inv;
    V3 clo, chi;   // offsets of the lo and hi planes
};

__device__ __forceinline__ float fast_shift(float p, bool up) {
    const float m = fabsf(p) * 0x1p-20f;
    return up ? p + m : p - m;
}

__device__ __forceinline__ FastRay fast_ray(const Ray &r) {
    FastRay f;
    const float e = 1e-20f;
    const float dx = fabsf(r.d.x) < e ? copysignf(e, r.d.x) : r.d.x;
    const float dy = fabsf(r.d.y) < e ? copysignf(e, r.d.y) : r.d.y;
    const float dz = fabsf(r.d.z) < e ? copysignf(e, r.d.z) : r.d.z;
    f.inv = V3{1.0f / dx, 1.0f / dy, 1.0f / dz};
    const float px = r.o.x * f.inv.x, py = r.o.y * f.inv.y, pz = r.o.z * f.inv.z;
    // the lo plane is the entry plane when inv >= 0: its offset moves up (distance down)
    f.clo = V3{fast_shift(px, f.inv.x >= 0.0f), fast_shift(py, f.inv.y >= 0.0f), fast_shift(pz, f.inv.z >= 0.0f)};
    f.chi = V3{fast_shift(px, f.inv.x < 0.0f), fast_shift(py, f.inv.y < 0.0f), fast_shift(pz, f.inv.z < 0.0f)};
    return f;
}

// true when the ray segment [0, tmax] may touch the box; tnear = entry distance (a lower bound)
__device__ __forceinline__ bool fast_slab(float4 lo, float4 hi, const FastRay &f, float tmax, float &tnear) {
    const float x1 = __fmaf_rn(lo.x, f.inv.x, -f.clo.x), x2 = __fmaf_rn(hi.x, f.inv.x, -f.chi.x);
    const float y1 = __fmaf_rn(lo.y, f.inv.y, -f.clo.y), y2 = __fmaf_rn(hi.y, f.inv.y, -f.chi.y);
    const float z1 = __fmaf_rn(lo.z, f.inv.z, -f.clo.z), z2 = __fmaf_rn(hi.z, f.inv.z, -f.chi.z);
    const float tn = fmaxf(fmaxf(fminf(x1, x2), fminf(y1, y2)), fmaxf(fminf(z1, z2), 0.0f));
    const float tf = fminf(fminf(fmaxf(x1, x2), fmaxf(y1, y2)), fminf(fmaxf(z1, z2), tmax));
    tnear = tn;
    return tn <= tf * 1.000001f;
}

struct FastCounts {
    uint32_t nodes;  // 32-byte node records fetched
    uint32_t tris;   // 48-byte triangle records fetched
};

template <bool kCount, class S>
__device__ __forceinline__ void fast_leaf(const S &s, const Ray &r, uint32_t first, uint32_t count,
                                          float &best_t, uint32_t &best_i, bool &have, FastCounts &cnt) {
    if (first + count > s.n_tri) { raise_error(s, MRT_ERR_LIMIT); return; }
    for (uint32_t k = first; k < first + count; ++k) {
        const float4 A = __ldg(&s.ftris[3 * k]);
        const float4 AB = __ldg(&s.ftris[3 * k + 1]);
        const float4 AC = __ldg(&s.ftris[3 * k + 2]);
        if (kCount) cnt.tris++;
        const uint32_t idx = __float_as_uint(A.w);
        if (r.exclude == hid(MRT_PRIM_TRIANGLE, idx)) continue;
        float t, u, v;
        if (!tri_test(v3(A), v3(AB), v3(AC), r, t, u, v)) continue;
        if (t < best_t || (t == best_t && idx < best_i)) {
            best_t = t;
            best_i = idx;
            have = true;
        }
    }
}


__device__ __forceinline__ void cmp_swap(float (&t)[kWide], uint32_t (&c)[kWide], int i, int j) {
    const bool sw = t[j] < t[i];
    const float ti = t[i], tj = t[j];
    const uint32_t ci = c[i], cj = c[j];
    t[i] = sw ? tj : ti;
    t[j] = sw ? ti : tj;
    c[i] = sw ? cj : ci;
    c[j] = sw ? ci : cj;
}

// One node of the FAST tree: kWide child records {min.xyz, a}{max.xyz, b} (b = 0: internal child,
// node a; b > 0: leaf of b triangles, a = its leaf code; b < 0: empty slot).  Returns the number of children the
// ray segment [0, tmax] may touch; with kSort their (entry distance, code) come first, nearest
// first, the others follow at +inf.
template <bool kSort, class S>
__device__ __forceinline__ int wide_children(const S &s, uint32_t node, const FastRay &f, float tmax,
                                             float (&t)[kWide], uint32_t (&c)[kWide]) {
    const float4 *p = s.fnodes + (size_t)node * (2 * kWide);
    float4 lo[kWide], hi[kWide];
#pragma unroll
    for (int k = 0; k < kWide; ++k) {
        lo[k] = __ldg(p + 2 * k);
        hi[k] = __ldg(p + 2 * k + 1);
    }
    int n = 0;
#pragma unroll
    for (int k = 0; k < kWide; ++k) {
        const int b = __float_as_int(hi[k].w);
        float tn;
        const bool hit = fast_slab(lo[k], hi[k], f, tmax, tn) && b >= 0;
        t[k] = hit ? tn : __int_as_float(0x7f800000);
        c[k] = __float_as_uint(lo[k].w);   // node index, or the leaf code written by the build
        n += hit ? 1 : 0;
    }
    if (kSort) {
        static_assert(kWide == 4, "sorting network for 4 children");
        cmp_swap(t, c, 0, 1);
        cmp_swap(t, c, 2, 3);
        cmp_swap(t, c, 0, 2);
        cmp_swap(t, c, 1, 3);
        cmp_swap(t, c, 1, 2);
    } else {
        // compact the hits to the front, order kept
#pragma unroll
        for (int k = 1; k < kWide; ++k)
#pragma unroll
            for (int m = k; m > 0; --m)
                if (t[m - 1] == __int_as_float(0x7f800000) && t[m] != __int_as_float(0x7f800000)) {
                    t[m - 1] = t[m]; t[m] = __int_as_float(0x7f800000);
                    const uint32_t x = c[m - 1]; c[m - 1] = c[m]; c[m] = x;
                }
    }
    return n;
}

template <class S>
__device__ __forceinline__ bool node_in_range(const S &s, uint32_t node) {
    return (uint64_t)(node + 1u) * kWide <= (uint64_t)s.n_fnodes;
}

// closest triangle with the reference's accept rule against the incoming length `len`: front to
// back, leaves as they are reached, entries beyond the best distance culled when popped
template <bool kCount = false>
__device__ bool fast_trace(const DevScene &s, const Ray &r, float &len, uint32_t &id, FastCounts *counts = nullptr) {
    if (s.n_tri == 0) return false;
    FastCounts cnt{0, 0};
    const FastRay f = fast_ray(r);
    float best_t = len;
    uint32_t best_i = 0;   // ties with a plane/sphere distance never win (index < 0 is impossible)
    bool have = false;
    uint32_t stack_n[kFastStack];
    float stack_t[kFastStack];
    int sp = 0;
    uint32_t cur = 0;      // the root node
    uint32_t steps = 0;
    for (;;) {
        if (cur == kNodeNone) {
            bool found = false;
            while (sp > 0) {
                --sp;
                if (stack_t[sp] <= best_t * 1.000001f) { cur = stack_n[sp]; found = true; break; }
            }
            if (!found) break;
        } else if (cur & kLeafCode) {
            fast_leaf<kCount>(s, r, code_first(cur), code_count(cur), best_t, best_i, have, cnt);
            cur = kNodeNone;
        } else {
            if (!node_in_range(s, cur) || ++steps > kMaxBvhSteps) { raise_error(s, MRT_ERR_LIMIT); break; }
            float ct[kWide];
            uint32_t cc[kWide];
            const int n = wide_children<true>(s, cur, f, best_t, ct, cc);
            if (kCount) cnt.nodes += kWide;
            cur = kNodeNone;
            if (n > 0) {
                if (sp + n - 1 > kFastStack) { raise_error(s, MRT_ERR_LIMIT); break; }
#pragma unroll
                for (int k = kWide - 1; k >= 1; --k)
                    if (k < n) { stack_n[sp] = cc[k]; stack_t[sp] = ct[k]; ++sp; }
                cur = cc[0];
            }
        }
    }
    if (counts) *counts = cnt;
    if (!have) return false;
    len = best_t;
    id = hid(MRT_PRIM_TRIANGLE, best_i);
    return true;
}

__device__ __forceinline__ bool fast_occ_leaf(const DevScene &s, const Ray &r, uint32_t first, uint32_t count,
                                              float dist) {
    if (first + count > s.n_tri) { raise_error(s, MRT_ERR_LIMIT); return false; }
    for (uint32_t k = first; k < first + count; ++k) {
        const float4 A = __ldg(&s.ftris[3 * k]);
        const float4 AB = __ldg(&s.ftris[3 * k + 1]);
        const float4 AC = __ldg(&s.ftris[3 * k + 2]);
        if (r.exclude == hid(MRT_PRIM_TRIANGLE, __float_as_uint(A.w))) continue;
        if (tri_occ(v3(A), v3(AB), v3(AC), r, dist)) return true;
    }
    return false;
}

__device__ inline bool fast_occ(const DevScene &s, const Ray &r, float dist) {
    if (s.n_tri == 0) return false;
    const FastRay f = fast_ray(r);
    uint32_t stack_n[kFastStack];
    int sp = 0;
    uint32_t cur = 0;
    uint32_t steps = 0;
    for (;;) {
        if (cur == kNodeNone) {
            if (sp == 0) return false;
            cur = stack_n[--sp];
        } else if (cur & kLeafCode) {
            if (fast_occ_leaf(s, r, code_first(cur), code_count(cur), dist)) return true;
            cur = kNodeNone;
        } else {
            if (!node_in_range(s, cur) || ++steps > kMaxBvhSteps) { raise_error(s, MRT_ERR_LIMIT); return false; }
            float ct[kWide];
            uint32_t cc[kWide];
            const int n = wide_children<false>(s, cur, f, dist, ct, cc);
            cur = kNodeNone;
            if (n > 0) {
                if (sp + n - 1 > kFastStack) { raise_error(s, MRT_ERR_LIMIT); return false; }
#pragma unroll
                for (int k = kWide - 1; k >= 1; --k)
                    if (k < n) stack_n[sp++] = cc[k];
                cur = cc[0];
            }
        }
    }
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
