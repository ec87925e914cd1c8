// mrt_grid.cu - RegularGrid<T> construction on the device.
//
// Bounds and size follow Shader::initializeAccelerators (Shader.cpp:40-113): the union of the
// primitive AABBs and the camera position, widened by Epsilon, and G = max(a*b, a) with
// a = N > 6 ? roundUpToPowerOf2(bitCounter(N)) : 2, b = roundUpToPowerOf2(bitCounter(a)) / 2.
// The fill restates RegularGrid::addPrimitives (RegularGrid.hpp:88-154): each primitive's
// candidate cell range from its AABB, then the primitive's own intersectBox against every
// candidate cell.  One thread per primitive counts, a scan gives the cell offsets, a second pass
// fills, and every cell's list is sorted by primitive index, which is the reference's insertion
// order (primitives are inserted in input order).
#include <algorithm>
#include <cfloat>

#include "mrt_internal.h"

using namespace mrt;
using namespace mrt_host;

namespace {

// intersectRayAABB lambda of Triangle::intersectBox, Triangle.cpp:155-219
__device__ bool edge_box(V3 orig, V3 vec, const Box &box) {
    float t_near = FLT_MIN, t_far = FLT_MAX;
    for (int k = 0; k < 3; ++k) {
        const float o = comp(orig, k), d = comp(vec, k);
        const float bmn = comp(box.mn, k), bmx = comp(box.mx, k);
        if (fabsf(d) < kEpsilon) {
            if ((o < bmn) || ((o + d) > bmx)) return false;
        } else {
            float t1 = (bmn - o) / d;
            float t2 = (bmx - o) / d;
            if (t1 > t2) { const float tmp = t1; t1 = t2; t2 = tmp; }
            t_near = smax(t1, t_near);
            t_far = smin(t2, t_far);
            if ((t_near > t_far) || (t_far < 0)) return false;
        }
    }
    return true;
}

// Triangle::intersectBox, Triangle.cpp:154-246
__device__ bool tri_in_box(V3 a, V3 ab, V3 ac, const Box &box) {
    const V3 vec = box.mx - box.mn;
    const bool iab = edge_box(a, ab, box);
    const bool iac = edge_box(a, ac, box);
    const V3 B = a + ab, C = a + ac;
    const bool ibc = edge_box(B, C - B, box);
    Ray r;
    r.o = box.mn;
    r.d = vec;
    r.depth = 1;
    r.exclude = MRT_HIT_NONE;
    float t, u, v;
    const bool iray = tri_test(a, ab, ac, r, t, u, v) && !(t >= kRayLengthMax);
    const V3 perp = cross(vec, ac);
    const bool inside = fabsf(dot(ab, perp)) < kEpsilon;
    return iab || iac || ibc || iray || inside;
}

// Sphere::intersectBox, Sphere.cpp:102-123
__device__ bool sph_in_box(float4 c, const Box &box) {
    float dmin = 0;
    const V3 ctr = v3(c);
    for (int k = 0; k < 3; ++k) {
        const float x = comp(ctr, k), a = comp(box.mn, k), b = comp(box.mx, k);
        if (x < a) dmin = dmin + (x - a) * (x - a);
        else if (x > b) dmin = dmin + (x - b) * (x - b);
    }
    return dmin <= c.w;
}

// Plane::distance / intersectBox, Plane.cpp:107-155
__device__ float pln_distance(V3 n, V3 o, V3 q) {
    const float d = n.x * -o.x + n.y * -o.y + n.z * -o.z;
    const float num = n.x * q.x + n.y * q.y + n.z * q.z + d;
    const float den = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
    return num / den;
}
__device__ bool pln_in_box(V3 n, V3 p, const Box &box) {
    const float dp = pln_distance(n, p, box.mx);
    const float dn = pln_distance(n, p, box.mn);
    return (dp <= 0 && dn >= 0) || (dp >= 0 && dn <= 0);
}

template <int T> __device__ Box prim_box(const DevScene &s, uint32_t i);
template <> __device__ Box prim_box<kTriangle>(const DevScene &s, uint32_t i) {   // Triangle.cpp:145-152
    const V3 A = v3(s.tri_a[i]), B = A + v3(s.tri_ab[i]), C = A + v3(s.tri_ac[i]);
    return Box{vmin(A, vmin(B, C)), vmax(A, vmax(B, C))};
}
template <> __device__ Box prim_box<kSphere>(const DevScene &s, uint32_t i) {   // Sphere.cpp:94-100
    const float4 c = s.sph[i];
    const float r = sqrtf(c.w);
    return Box{subs(v3(c), r), adds(v3(c), r)};
}
template <> __device__ Box prim_box<kPlane>(const DevScene &s, uint32_t i) {   // Plane.cpp:80-105
    const V3 n = v3(s.pln_n[i]), p = v3(s.pln_p[i]);
    V3 right{0, 0, 0};
    if (n.x >= 1) right = V3{0, 1, 1};
    else if (n.y >= 1) right = V3{1, 0, 1};
    else if (n.z >= 1) right = V3{1, 1, 0};
    else if (n.x <= -1) right = V3{0, 1, 1};
    else if (n.y <= -1) right = V3{1, 0, 1};
    else if (n.z <= -1) right = V3{1, 1, 0};
    right = normalize(right);
    return Box{p + right * -100.0f, p + right * 100.0f};
}

template <int T> __device__ bool prim_in_box(const DevScene &s, uint32_t i, const Box &b) {
    if (T == kTriangle) return tri_in_box(v3(s.tri_a[i]), v3(s.tri_ab[i]), v3(s.tri_ac[i]), b);
    if (T == kSphere) return sph_in_box(s.sph[i], b);
    return pln_in_box(v3(s.pln_n[i]), v3(s.pln_p[i]), b);
}

struct GridBuildParams {
    int32_t G;
    V3 mn;
    float sx, sy, sz, dx, dy, dz, rx, ry, rz;
};

__device__ __forceinline__ void cell_range(float lo, float hi, float mn, float r, float size, int32_t G, int32_t &c1,
                                           int32_t &c2) {
    c1 = f2i_x86((lo - mn) * r);
    c2 = f2i_x86((hi - mn) * r) + 1;
    c1 = c1 > 0 ? c1 : 0;
    c2 = (G - 1 < c2) ? G - 1 : c2;
    c2 = fabsf(size) < kEpsilon ? 0 : c2;
    c1 = (c2 < c1) ? c2 : c1;
}

// pass 0 counts references per cell, pass 1 writes them
template <int T, int PASS>
__global__ void k_grid_fill(DevScene s, GridBuildParams p, uint32_t n, uint32_t *count, const uint32_t *start,
                            uint32_t *fill, uint32_t *refs) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Box bd = prim_box<T>(s, i);
    int32_t x1, x2, y1, y2, z1, z2;
    cell_range(bd.mn.x, bd.mx.x, p.mn.x, p.rx, p.sx, p.G, x1, x2);
    cell_range(bd.mn.y, bd.mx.y, p.mn.y, p.ry, p.sy, p.G, y1, y2);
    cell_range(bd.mn.z, bd.mx.z, p.mn.z, p.rz, p.sz, p.G, z1, z2);
    // a NaN or out-of-range box gives negative cell indices, which the reference would index with
    // (undefined behaviour); such a primitive is left out of the grid
    if (x1 < 0 || y1 < 0 || z1 < 0 || x2 < 0 || y2 < 0 || z2 < 0) return;
    for (int32_t x = x1; x <= x2; ++x)
        for (int32_t y = y1; y <= y2; ++y)
            for (int32_t z = z1; z <= z2; ++z) {
                const size_t idx = (size_t)x + (size_t)y * (size_t)p.G + (size_t)z * (size_t)p.G * (size_t)p.G;
                const V3 pos{p.mn.x + (float)x * p.dx, p.mn.y + (float)y * p.dy, p.mn.z + (float)z * p.dz};
                const Box cell{pos, pos + V3{p.dx, p.dy, p.dz}};
                if (!prim_in_box<T>(s, i, cell)) continue;
                if (PASS == 0) atomicAdd(&count[idx], 1u);
                else refs[start[idx] + atomicAdd(&fill[idx], 1u)] = i;
            }
}

__global__ void k_sort_cells(uint64_t ncell, const uint32_t *start, uint32_t *refs) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const uint32_t b = start[c], e = start[c + 1];
    for (uint32_t i = b + 1; i < e; ++i) {
        const uint32_t v = refs[i];
        uint32_t j = i;
        while (j > b && refs[j - 1] > v) { refs[j] = refs[j - 1]; --j; }
        refs[j] = v;
    }
}

// exclusive scan of counts into start (ncell + 1 entries), three-level
__global__ void k_block_sums(const uint32_t *in, uint64_t n, uint32_t *sums, uint32_t per) {
    const uint64_t b = (uint64_t)blockIdx.x * per;
    uint32_t s = 0;
    for (uint64_t i = b + threadIdx.x; i < b + per && i < n; i += blockDim.x) s += in[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    __shared__ uint32_t w[32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += w[k];
        sums[blockIdx.x] = t;
    }
}
__global__ void k_block_scan_write(const uint32_t *in, uint64_t n, const uint32_t *offsets, uint32_t per, uint32_t *out) {
    if (threadIdx.x != 0) return;
    const uint64_t b = (uint64_t)blockIdx.x * per;
    uint32_t acc = offsets[blockIdx.x];
    for (uint64_t i = b; i < b + per && i < n; ++i) { out[i] = acc; acc += in[i]; }
    if (b + per >= n && b < n) out[n] = acc;
}

uint32_t bit_counter(uint32_t n) { uint32_t c = 0; while (n > 0) { ++c; n >>= 1; } return c; }   // Utils.cpp:26-33
uint32_t round_up_pow2(uint32_t v) {   // Utils.cpp:15-24
    --v; v |= v >> 1u; v |= v >> 2u; v |= v >> 4u; v |= v >> 8u; v |= v >> 16u; ++v; return v;
}
int32_t grid_size_rule(uint32_t n) {   // Shader.cpp:76-105
    const int32_t a = n > 6 ? (int32_t)round_up_pow2(bit_counter(n)) : 2;
    const int32_t b = (int32_t)(round_up_pow2(bit_counter((uint32_t)a)) / 2);
    return std::max(a * b, a);
}

struct HostBox {
    V3 mn, mx;
};

HostBox host_prim_box(const MrtScene *s, int type, uint32_t i) {
    if (type == kTriangle) {
        const float *p = &s->h_abc[9ull * i];
        const V3 A{p[0], p[1], p[2]};
        const V3 ab = V3{p[3], p[4], p[5]} - A, ac = V3{p[6], p[7], p[8]} - A;
        const V3 B = A + ab, C = A + ac;
        return HostBox{vmin(A, vmin(B, C)), vmax(A, vmax(B, C))};
    }
    if (type == kSphere) {
        const float *c = &s->h_sph[4ull * i];
        const float r = sqrtf(c[3]);
        return HostBox{subs(V3{c[0], c[1], c[2]}, r), adds(V3{c[0], c[1], c[2]}, r)};
    }
    const float *p = &s->h_pln[6ull * i];
    const V3 n{p[3], p[4], p[5]}, pt{p[0], p[1], p[2]};
    V3 right{0, 0, 0};
    if (n.x >= 1) right = V3{0, 1, 1};
    else if (n.y >= 1) right = V3{1, 0, 1};
    else if (n.z >= 1) right = V3{1, 1, 0};
    else if (n.x <= -1) right = V3{0, 1, 1};
    else if (n.y <= -1) right = V3{1, 0, 1};
    else if (n.z <= -1) right = V3{1, 1, 0};
    right = normalize(right);
    return HostBox{pt + right * -100.0f, pt + right * 100.0f};
}

template <int T>
void launch_fill(MrtScene *s, const GridBuildParams &p, uint32_t n, uint32_t *count, const uint32_t *start, uint32_t *fill,
                 uint32_t *refs, int pass) {
    if (n == 0) return;
    const uint32_t g = (n + 127) / 128;
    if (pass == 0) k_grid_fill<T, 0><<<g, 128, 0, s->ctx->stream>>>(s->dev, p, n, count, start, fill, refs);
    else k_grid_fill<T, 1><<<g, 128, 0, s->ctx->stream>>>(s->dev, p, n, count, start, fill, refs);
}

}  // namespace

// the triangle grid's packed records: A, AB, AC in 9 of 16 floats (one 64-byte record per triangle, read
// by the walk with one 256-bit and one 32-bit load instead of three 128-bit loads from three arrays:
// 285 -> 322 Mrays/s on the 1080p soup frame at G = 128)
#ifndef MRT_GRID_TRIREC
#define MRT_GRID_TRIREC 1
#endif
constexpr bool kGridTriRecords = MRT_GRID_TRIREC != 0;
__global__ void k_pack_trec(uint32_t n, const float4 *__restrict__ a, const float4 *__restrict__ ab,
                            const float4 *__restrict__ ac, float *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 A = a[i], B = ab[i], C = ac[i];
    float4 *r = reinterpret_cast<float4 *>(out + 16 * (size_t)i);
    r[0] = make_float4(A.x, A.y, A.z, B.x);
    r[1] = make_float4(B.y, B.z, C.x, C.y);
    r[2] = make_float4(C.z, 0.0f, 0.0f, 0.0f);
    r[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

namespace mrt_host {

int build_grids(MrtScene *s, const float *cam_min, const float *cam_max, int grid_size, int grid_index) {
    MrtContext *ctx = s->ctx;
    cudaStream_t q = ctx->stream;
    for (int type = 0; type < 3; ++type) {
        const uint32_t n = type == kTriangle ? s->n_tri : (type == kSphere ? s->n_sph : s->n_pln);
        // Scene::getBounds (Scene.cpp:42-45) over the primitives, then the camera (Camera.cpp:39-44)
        V3 mn{kRayLengthMax, kRayLengthMax, kRayLengthMax}, mx{-kRayLengthMax, -kRayLengthMax, -kRayLengthMax};
        for (uint32_t i = 0; i < n; ++i) {
            const HostBox b = host_prim_box(s, type, i);
            mn = vmin(b.mn, mn);
            mx = vmax(b.mx, mx);
        }
        mn = vmin(V3{cam_min[0], cam_min[1], cam_min[2]}, mn);
        mx = vmax(V3{cam_max[0], cam_max[1], cam_max[2]}, mx);
        const V3 bmn = subs(mn, kEpsilon), bmx = adds(mx, kEpsilon);
        int32_t G = grid_size_rule(n);
        if (type == kTriangle && grid_size > 0) G = grid_size;
        const uint64_t ncell = (uint64_t)G * G * G;
        // RegularGrid ctor, RegularGrid.hpp:50-67
        DevGrid &g = s->dev.grid[type];
        g.G = G;
        g.shift = bit_counter((uint32_t)G) - 1;
        g.index_mode = grid_index;
        g.has = n > 0;
        g.mn = bmn;
        g.mx = bmx;
        const V3 size = bmx - bmn;
        g.sr = V3{(float)G / size.x, (float)G / size.y, (float)G / size.z};
        g.cw = size * (1.0f / (float)G);
        GridBuildParams p;
        p.G = G;
        p.mn = bmn;
        p.sx = bmx.x - bmn.x; p.sy = bmx.y - bmn.y; p.sz = bmx.z - bmn.z;
        p.dx = p.sx / (float)G; p.dy = p.sy / (float)G; p.dz = p.sz / (float)G;
        p.rx = p.dx > 0 ? 1.0f / p.dx : 1.0f;
        p.ry = p.dy > 0 ? 1.0f / p.dy : 1.0f;
        p.rz = p.dz > 0 ? 1.0f / p.dz : 1.0f;
        int st = dev_alloc(ctx, s->grid_start[type], 4ull * (ncell + 1));
        DevBuf count, fill, sums, offs;
        const uint32_t per = 8192;
        const uint64_t nblk = (ncell + per - 1) / per;
        if (st == MRT_OK) st = dev_alloc(ctx, count, 4ull * ncell);
        if (st == MRT_OK) st = dev_alloc(ctx, fill, 4ull * ncell);
        if (st == MRT_OK) st = dev_alloc(ctx, sums, 4ull * nblk + 4);
        if (st == MRT_OK) st = dev_alloc(ctx, offs, 4ull * nblk + 4);
        if (st == MRT_OK) {
            cudaMemsetAsync(count.ptr, 0, 4ull * ncell, q);
            cudaMemsetAsync(fill.ptr, 0, 4ull * ncell, q);
            if (type == kTriangle) launch_fill<kTriangle>(s, p, n, (uint32_t *)count.ptr, nullptr, nullptr, nullptr, 0);
            else if (type == kSphere) launch_fill<kSphere>(s, p, n, (uint32_t *)count.ptr, nullptr, nullptr, nullptr, 0);
            else launch_fill<kPlane>(s, p, n, (uint32_t *)count.ptr, nullptr, nullptr, nullptr, 0);
            k_block_sums<<<(uint32_t)nblk, 256, 0, q>>>((const uint32_t *)count.ptr, ncell, (uint32_t *)sums.ptr, per);
            std::vector<uint32_t> hs(nblk), ho(nblk);
            st = cuda_status(ctx, cudaMemcpyAsync(hs.data(), sums.ptr, 4ull * nblk, cudaMemcpyDeviceToHost, q), "grid sums");
            if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "grid count");
            uint64_t total = 0;
            for (uint64_t b = 0; b < nblk; ++b) { ho[b] = (uint32_t)total; total += hs[b]; }
            if (st == MRT_OK && total > 0xFFFFFFF0ull) { set_error(ctx, "grid: more than 2^32 references"); st = MRT_ERR_LIMIT; }
            if (st == MRT_OK) st = cuda_status(ctx, cudaMemcpyAsync(offs.ptr, ho.data(), 4ull * nblk, cudaMemcpyHostToDevice, q), "grid offs");
            if (st == MRT_OK) {
                k_block_scan_write<<<(uint32_t)nblk, 32, 0, q>>>((const uint32_t *)count.ptr, ncell, (const uint32_t *)offs.ptr,
                                                                per, (uint32_t *)s->grid_start[type].ptr);
                st = dev_alloc(ctx, s->grid_refs[type], 4ull * (total ? total : 1));
            }
            if (st == MRT_OK) {
                const uint32_t *start = (const uint32_t *)s->grid_start[type].ptr;
                uint32_t *refs = (uint32_t *)s->grid_refs[type].ptr;
                if (type == kTriangle) launch_fill<kTriangle>(s, p, n, nullptr, start, (uint32_t *)fill.ptr, refs, 1);
                else if (type == kSphere) launch_fill<kSphere>(s, p, n, nullptr, start, (uint32_t *)fill.ptr, refs, 1);
                else launch_fill<kPlane>(s, p, n, nullptr, start, (uint32_t *)fill.ptr, refs, 1);
                k_sort_cells<<<(uint32_t)((ncell + 255) / 256), 256, 0, q>>>(ncell, start, refs);
                st = cuda_status(ctx, cudaGetLastError(), "grid kernels");
                if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "grid build");
                s->grid_refs_count[type] = total;
            }
        }
        dev_free(count); dev_free(fill); dev_free(sums); dev_free(offs);
        if (st != MRT_OK) return st;
        g.start = (const uint32_t *)s->grid_start[type].ptr;
        g.refs = (const uint32_t *)s->grid_refs[type].ptr;
        g.trec = nullptr;
        if (type == kTriangle && n > 0 && kGridTriRecords) {
            st = dev_alloc(ctx, s->grid_trec, 64ull * n);
            if (st != MRT_OK) return st;
            k_pack_trec<<<(n + 255) / 256, 256, 0, q>>>(n, s->dev.tri_a, s->dev.tri_ab, s->dev.tri_ac, (float *)s->grid_trec.ptr);
            st = cuda_status(ctx, cudaGetLastError(), "grid records");
            if (st != MRT_OK) return st;
            g.trec = (const float *)s->grid_trec.ptr;
        }
    }
    return MRT_OK;
}

}  // namespace mrt_host
