// mrt_bvh.cu - BVH construction.
//
// REFERENCE tree: BVH<T>::BVH + build + getSplitIndex_SAH (BVH.hpp:64-155, 273-311) restated on the
// host with the same float operations and node numbering, then uploaded.  The reference never
// reorders primitives, so leaf offsets index the input arrays.
//
// FAST tree: built on the device.  Triangle boxes padded outward -> 30-bit Morton codes of the
// centroids -> stable LSD radix sort (own kernels) -> Karras' parallel hierarchy ("Maximizing
// parallelism in the construction of BVHs, octrees and k-d trees", HPG 2012) -> bottom-up box fit
// -> records in child-pair layout (32 bytes per record), subtrees of <= leaf_max_setting() (at most 3)
// triangles collapsed into leaves where the surface-area cost says so -> the binary tree collapsed
// into 8-wide nodes with 16-bit quantised child boxes (128 bytes: one cache line per traversal step;
// each wide node opens the largest internal children of a binary node until it holds 8), children
// placed in slots by octant, internal children numbered consecutively, the leaf children's triangles
// copied to consecutive 48-byte records.  A traversal step of the 8-wide tree replaces about three of
// the binary tree's, shortening the chain of dependent node fetches per ray.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "mrt_internal.h"

using namespace mrt;
using namespace mrt_host;

namespace {

// ============================== reference tree (host) =======================================
struct HBox {
    V3 mn, mx;
};

HBox hunion(const HBox &b1, const HBox &b2) { return HBox{vmin(b1.mn, b2.mn), vmax(b1.mx, b2.mx)}; }   // AABB.cpp:52-60
float harea(const HBox &b) {   // AABB.cpp:37-49
    const float lx = b.mx.x - b.mn.x, ly = b.mx.y - b.mn.y, lz = b.mx.z - b.mn.z;
    const float bt = 2 * lx * lz, xy = 2 * lx * ly, zy = 2 * lz * ly;
    return bt + xy + zy;
}

uint32_t sah_split(const HBox *boxes, uint32_t N, std::vector<float> &la, std::vector<float> &ra) {
    const uint32_t L = 2;
    la.assign(N - L, 0.0f);
    ra.assign(N - L, 0.0f);
    HBox lb = boxes[0];
    la[0] = harea(lb);
    for (uint32_t i = 1; i < N - L; ++i) { lb = hunion(lb, boxes[i]); la[i] = harea(lb); }
    HBox rb = boxes[N - 1];
    ra[N - L - 1] = harea(rb);
    for (uint32_t i = N - 2; i > L; --i) { rb = hunion(rb, boxes[i]); ra[i - L] = harea(rb); }
    uint32_t split = L;
    float min_sah = (float)L * la[L - 1] + (float)(N - L) * ra[L - 1];
    for (uint32_t i = L; i < N - L; ++i) {
        const float sl = (float)(i + 1) * la[i];
        const float sr = (float)(N - (i + 1)) * ra[i];
        const float sah = sl + sr;
        if (sah < min_sah) { split = i + 1; min_sah = sah; }
    }
    return split;
}

std::vector<RefNode> ref_build(const std::vector<HBox> &pboxes) {
    const uint32_t N = (uint32_t)pboxes.size();
    if (N == 0) return std::vector<RefNode>(1, RefNode{{0, 0, 0}, {0, 0, 0}, 0, 0});
    std::vector<RefNode> nodes(2 * (size_t)N - 1, RefNode{{0, 0, 0}, {0, 0, 0}, 0, 0});
    std::vector<HBox> boxes(N);
    std::vector<float> la, ra;
    uint32_t st_id[512] = {0}, st_b[512] = {0}, st_e[512] = {0};
    uint32_t sp = 1, id = 0, begin = 0, end = N, max_id = 0;
    do {
        HBox nb = pboxes[begin];
        boxes[0] = nb;
        const uint32_t size = end - begin;
        for (uint32_t i = begin + 1; i < end; ++i) {
            nb = hunion(pboxes[i], nb);
            boxes[i - begin] = pboxes[i];
        }
        RefNode &nd = nodes[id];
        nd.mn[0] = nb.mn.x; nd.mn[1] = nb.mn.y; nd.mn[2] = nb.mn.z;
        nd.mx[0] = nb.mx.x; nd.mx[1] = nb.mx.y; nd.mx[2] = nb.mx.z;
        if (size <= 2) {
            nd.offset = begin;
            nd.count = size;
            --sp; id = st_id[sp]; begin = st_b[sp]; end = st_e[sp];
        } else {
            const uint32_t left = max_id + 1, right = left + 1;
            nd.offset = left;
            max_id = std::max(right, max_id);
            const uint32_t split = size <= 4 ? 2 : sah_split(boxes.data(), size, la, ra);
            if (sp >= 512) break;   // the reference's fixed 512-entry stack (BVH.hpp:93-95)
            st_id[sp] = right; st_b[sp] = begin + split; st_e[sp] = end; ++sp;
            id = left;
            end = begin + split;
        }
    } while (sp > 0);
    nodes.resize(max_id + 1);
    return nodes;
}

// ============================== FAST tree (device) ===========================================
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;

__device__ __forceinline__ uint32_t float_key(float f) {   // order-preserving float -> uint
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float_(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// padded triangle boxes (min.xyz, max.xyz as two float4) and the centroid bounds
__global__ void k_tri_boxes(uint32_t n, const float4 *__restrict__ a4, const float4 *__restrict__ ab4,
                            const float4 *__restrict__ ac4, float4 *bmin, float4 *bmax, uint32_t *cbounds) {
    __shared__ uint32_t smin[3][32], smax[3][32];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float c[3] = {0, 0, 0};
    bool valid = i < n;
    if (valid) {
        const V3 A = v3(a4[i]), ab = v3(ab4[i]), ac = v3(ac4[i]);
        const V3 B = A + ab, C = A + ac;
        V3 mn = vmin(A, vmin(B, C)), mx = vmax(A, vmax(B, C));
        const float m = fmaxf(fmaxf(fmaxf(fabsf(mn.x), fabsf(mx.x)), fmaxf(fabsf(mn.y), fabsf(mx.y))),
                              fmaxf(fabsf(mn.z), fabsf(mx.z)));
        const float e = fmaxf(fmaxf(mx.x - mn.x, mx.y - mn.y), mx.z - mn.z);
        const float pad = 4e-6f * m + 2e-5f * e + 1e-30f;
        mn = subs(mn, pad);
        mx = adds(mx, pad);
        bmin[i] = make_float4(mn.x, mn.y, mn.z, 0.0f);
        bmax[i] = make_float4(mx.x, mx.y, mx.z, 0.0f);
        c[0] = 0.5f * (mn.x + mx.x); c[1] = 0.5f * (mn.y + mx.y); c[2] = 0.5f * (mn.z + mx.z);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 3; ++k) {
        uint32_t lo = valid ? float_key(c[k]) : 0xFFFFFFFFu, hi = valid ? float_key(c[k]) : 0u;
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
        }
        if (lane == 0) { smin[k][warp] = lo; smax[k][warp] = hi; }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int k = threadIdx.x;
        uint32_t lo = 0xFFFFFFFFu, hi = 0u;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { lo = min(lo, smin[k][w]); hi = max(hi, smax[k][w]); }
        atomicMin(&cbounds[k], lo);
        atomicMax(&cbounds[3 + k], hi);
    }
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {   // 10 bits -> every third bit
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_morton(uint32_t n, const float4 *__restrict__ bmin, const float4 *__restrict__ bmax,
                         const uint32_t *__restrict__ cbounds, uint32_t *keys, uint32_t *vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 lo = bmin[i], hi = bmax[i];
    float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
        const float mn = key_float_(cbounds[k]), mx = key_float_(cbounds[3 + k]);
        const float ext = mx - mn;
        float u = ext > 0.0f ? (c[k] - mn) / ext : 0.5f;
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        q[k] = min((uint32_t)(u * 1024.0f), 1023u);
    }
    keys[i] = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
    vals[i] = i;
}

// --- stable LSD radix sort, 8-bit digits --------------------------------------------------------
__global__ void k_rs_hist(const uint32_t *__restrict__ keys, uint32_t n, int shift, uint32_t *hist, uint32_t nblocks) {
    __shared__ uint32_t cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t e = base + r * kSortThreads + threadIdx.x;
        if (e < n) atomicAdd(&cnt[(keys[e] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

// exclusive scan of m values in place, one block of 1024 threads
__global__ void k_scan_exclusive(uint32_t *data, uint32_t m) {
    __shared__ uint32_t part[1024];
    const uint32_t per = (m + 1023) / 1024;
    const uint32_t b = threadIdx.x * per, e = min(b + per, m);
    uint32_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += data[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const uint32_t v = threadIdx.x >= (uint32_t)o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t acc = part[threadIdx.x] - s;
    for (uint32_t i = b; i < e; ++i) { const uint32_t v = data[i]; data[i] = acc; acc += v; }
}

__global__ void k_rs_scatter(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint32_t *kout,
                             uint32_t *vout, uint32_t n, int shift, const uint32_t *__restrict__ hist, uint32_t nblocks) {
    __shared__ uint32_t base[256], running[256], total[256];
    __shared__ uint32_t wcnt[kSortThreads / 32][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    base[tid] = hist[tid * nblocks + blockIdx.x];
    running[tid] = 0;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int r = 0; r < kSortItems; ++r) {
        for (int w = 0; w < kSortThreads / 32; ++w) wcnt[w][tid] = 0;
        __syncthreads();
        const uint32_t e = blockIdx.x * kSortTile + r * kSortThreads + tid;
        const bool valid = e < n;
        uint32_t key = 0, val = 0, d = 256;
        if (valid) { key = kin[e]; val = vin[e]; d = (key >> shift) & 255u; }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t rank = __popc(peers & lt_mask);
        if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        {
            uint32_t acc = 0;
            for (int w = 0; w < kSortThreads / 32; ++w) { const uint32_t c = wcnt[w][tid]; wcnt[w][tid] = acc; acc += c; }
            total[tid] = acc;
        }
        __syncthreads();
        if (valid) {
            const uint32_t pos = base[d] + running[d] + wcnt[warp][d] + rank;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        running[tid] += total[tid];
    }
}

// --- Karras hierarchy --------------------------------------------------------------------------
__device__ __forceinline__ int kdelta(const uint32_t *keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = keys[i], b = keys[j];
    if (a == b) return 32 + __clz((uint32_t)(i ^ j));
    return __clz(a ^ b);
}

constexpr uint32_t kLeafBit = 0x80000000u;

__global__ void k_karras(int n, const uint32_t *__restrict__ keys, uint32_t *left, uint32_t *right, uint32_t *first,
                         uint32_t *last, uint32_t *parent_int, uint32_t *parent_leaf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = kdelta(keys, n, i, i - d);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = kdelta(keys, n, i, j);
    int s = 0;
    for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
        if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    const int gamma = i + s * d + min(d, 0);
    const int f = min(i, j), la = max(i, j);
    const uint32_t lc = (f == gamma) ? (kLeafBit | (uint32_t)gamma) : (uint32_t)gamma;
    const uint32_t rc = (la == gamma + 1) ? (kLeafBit | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
    left[i] = lc;
    right[i] = rc;
    first[i] = (uint32_t)f;
    last[i] = (uint32_t)la;
    if (lc & kLeafBit) parent_leaf[lc & ~kLeafBit] = (uint32_t)i; else parent_int[lc] = (uint32_t)i;
    if (rc & kLeafBit) parent_leaf[rc & ~kLeafBit] = (uint32_t)i; else parent_int[rc] = (uint32_t)i;
}

__device__ __forceinline__ void child_box(uint32_t c, const uint32_t *__restrict__ vals, const float4 *bmin,
                                          const float4 *bmax, const float4 *imin, const float4 *imax, float4 &lo,
                                          float4 &hi) {
    if (c & kLeafBit) {
        const uint32_t t = vals[c & ~kLeafBit];
        lo = bmin[t];
        hi = bmax[t];
    } else {
        lo = __ldcg(&imin[c]);
        hi = __ldcg(&imax[c]);
    }
}

__global__ void k_fit(int n, const uint32_t *__restrict__ vals, const float4 *__restrict__ bmin,
                      const float4 *__restrict__ bmax, const uint32_t *__restrict__ left, const uint32_t *__restrict__ right,
                      const uint32_t *__restrict__ parent_int, const uint32_t *__restrict__ parent_leaf, uint32_t *counter,
                      float4 *imin, float4 *imax) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t node = parent_leaf[j];
    for (int guard = 0; guard < 4096 && node < (uint32_t)(n - 1); ++guard) {
        __threadfence();
        if (atomicAdd(&counter[node], 1u) == 0u) return;   // the other child is not ready yet
        float4 l0, l1, r0, r1;
        child_box(left[node], vals, bmin, bmax, imin, imax, l0, l1);
        child_box(right[node], vals, bmin, bmax, imin, imax, r0, r1);
        __stcg(&imin[node], make_float4(fminf(l0.x, r0.x), fminf(l0.y, r0.y), fminf(l0.z, r0.z), 0.0f));
        __stcg(&imax[node], make_float4(fmaxf(l1.x, r1.x), fmaxf(l1.y, r1.y), fmaxf(l1.z, r1.z), 0.0f));
        if (node == 0) return;
        node = parent_int[node];
    }
}

__device__ __forceinline__ void write_record(float4 *rec, float4 lo, float4 hi, uint32_t a, uint32_t b) {
    rec[0] = make_float4(lo.x, lo.y, lo.z, __uint_as_float(a));
    rec[1] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(b));
}

__device__ __forceinline__ float half_area(float4 lo, float4 hi) {
    const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    return dx * dy + dy * dz + dz * dx;
}

// --- leaf choice -------------------------------------------------------------------------------
// A subtree of at most leaf_max triangles becomes one leaf when that is cheaper by the surface-area
// cost model than keeping its inner nodes.  Per ray that reaches the subtree's box, a leaf costs
// kTriCost per triangle; an inner node costs kNodeCost plus its two children's costs, each weighted
// by the share of the node's box area its box has.  The unit is one box test: 2.2 box tests per
// triangle test and 2 per opened inner node fit the frame times of the 1,000,000-triangle soup at
// leaves of 1, 2 and 3 triangles, and still do for the 8-wide tree (node cost 1 or triangle cost 4:
// equal; node cost 4: -11 % on the soup frame, triangle cost 1.2: -6 %; the terrain PathTracer within
// 0.2 % except node cost 4 and triangle cost 1.2, -3 %).  Scattered small triangles (the soups) end up one per leaf: two
// boxes cull better than two triangle tests; touching triangles (a heightfield) stay in pairs.
#ifndef MRT_BVH_TRI_COST
#define MRT_BVH_TRI_COST 2.2f
#endif
#ifndef MRT_BVH_NODE_COST
#define MRT_BVH_NODE_COST 2.0f
#endif
constexpr float kTriCost = MRT_BVH_TRI_COST, kNodeCost = MRT_BVH_NODE_COST;
constexpr int kLeafCostDepth = 3;   // inner levels of a subtree of up to 4 triangles

struct BinView {
    const uint32_t *vals;
    const float4 *bmin, *bmax;
    const uint32_t *left, *right, *first, *last;
    const float4 *imin, *imax;
    __device__ void box(uint32_t c, float4 &lo, float4 &hi) const {
        if (c & kLeafBit) {
            const uint32_t t = vals[c & ~kLeafBit];
            lo = bmin[t];
            hi = bmax[t];
        } else {
            lo = imin[c];
            hi = imax[c];
        }
    }
    __device__ uint32_t count(uint32_t c) const { return (c & kLeafBit) ? 1u : last[c] - first[c] + 1u; }
};

template <int D>
__device__ float subtree_cost(const BinView &v, uint32_t c);

template <int D>
__device__ float split_cost(const BinView &v, uint32_t c) {
    float4 lo, hi;
    v.box(c, lo, hi);
    const float a = half_area(lo, hi);
    float cost = kNodeCost;
    const uint32_t ch[2] = {v.left[c], v.right[c]};
    for (int k = 0; k < 2; ++k) {
        float4 l2, h2;
        v.box(ch[k], l2, h2);
        const float share = a > 0.0f ? half_area(l2, h2) / a : 1.0f;
        cost += share * subtree_cost<D - 1>(v, ch[k]);
    }
    return cost;
}

template <int D>
__device__ float subtree_cost(const BinView &v, uint32_t c) {
    if (c & kLeafBit) return kTriCost;
    const float leaf = kTriCost * (float)v.count(c);
    if constexpr (D == 0) return leaf;
    else return fminf(leaf, split_cost<D>(v, c));
}

// inner node c (count <= leaf_max) as one leaf?
__device__ __forceinline__ bool leaf_by_cost(const BinView &v, uint32_t c) {
    return kTriCost * (float)v.count(c) <= split_cost<kLeafCostDepth>(v, c);
}

// one record per child of every internal node (pair at 2 + 2k), plus the root record 0
__global__ void k_emit(int n, int leaf_max, const uint32_t *__restrict__ vals, const float4 *__restrict__ bmin,
                       const float4 *__restrict__ bmax, const uint32_t *__restrict__ left, const uint32_t *__restrict__ right,
                       const uint32_t *__restrict__ first, const uint32_t *__restrict__ last, const float4 *__restrict__ imin,
                       const float4 *__restrict__ imax, float4 *records) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n - 1) return;
    const BinView v{vals, bmin, bmax, left, right, first, last, imin, imax};
    if (k == 0) {
        const uint32_t cnt = last[0] - first[0] + 1;
        if ((int)cnt <= leaf_max && leaf_by_cost(v, 0u)) write_record(records, imin[0], imax[0], first[0], cnt);
        else write_record(records, imin[0], imax[0], 2u, 0u);
        write_record(records + 2, make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0), 0u, 0u);
    }
    for (int side = 0; side < 2; ++side) {
        const uint32_t c = side == 0 ? left[k] : right[k];
        float4 *rec = records + 2 * (2 + 2 * (size_t)k + side);
        float4 lo, hi;
        if (c & kLeafBit) {
            const uint32_t j = c & ~kLeafBit;
            lo = bmin[vals[j]];
            hi = bmax[vals[j]];
            write_record(rec, lo, hi, j, 1u);
        } else {
            lo = imin[c];
            hi = imax[c];
            const uint32_t cnt = last[c] - first[c] + 1;
            if ((int)cnt <= leaf_max && leaf_by_cost(v, c)) write_record(rec, lo, hi, first[c], cnt);
            else write_record(rec, lo, hi, 2u + 2u * c, 0u);
        }
    }
}

__global__ void k_leaf_tris(uint32_t n, const uint32_t *__restrict__ vals, const float4 *__restrict__ a4,
                            const float4 *__restrict__ ab4, const float4 *__restrict__ ac4, float4 *out) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t t = vals[j];
    const float4 a = a4[t];
    out[3 * (size_t)j] = make_float4(a.x, a.y, a.z, __uint_as_float(t));
    out[3 * (size_t)j + 1] = ab4[t];
    out[3 * (size_t)j + 2] = ac4[t];
}

__global__ void k_single_leaf(const float4 *bmin, const float4 *bmax, float4 *records) {
    write_record(records, bmin[0], bmax[0], 0u, 1u);
}

// ------------------------------ binary -> 8-wide compressed nodes ------------------------------
// Each wide node starts from the children of one binary internal node (or from the root record) and
// opens its largest-area internal child until it holds kWide children.  Its box is the union of the
// children's boxes; per axis the children's planes are quantised on a grid p + 2^E q (16-bit q,
// lo rounded down and hi up, so every quantised box contains the exact one), the children are
// placed in slots by the octant of their centre within the node, internal children get consecutive
// node indices (one allocation per node), and the triangles of the leaf children are copied to
// consecutive records (one allocation per node).  One launch per level of the wide tree.
struct CollapseItem {
    uint32_t rec;     // first seed record: the root record 0 (one seed) or a child pair 2 + 2k (two seeds)
    uint32_t seeds;   // 1 or 2
    uint32_t node;    // the wide node it becomes
};

__device__ __forceinline__ bool rec_internal(const float4 *bin, uint32_t r) { return __float_as_int(bin[2 * (size_t)r + 1].w) == 0; }

// grid step exponent E of one axis (2^E >= extent / 65534)
__device__ __forceinline__ int grid_exponent(float lo, float hi) {
    const double want = ((double)hi - (double)lo) / 65534.0;
    if (!(want > 0x1p-126)) return -126;
    int ex = 0;
    const double m = frexp(want, &ex);   // want = m 2^ex, m in [0.5, 1)
    return m == 0.5 ? ex - 1 : ex;
}
// a child's planes on the grid, lo rounded down and hi up (with a 2^-20 step guard against the
// rounding of the double-precision subtraction), as lo | hi << 16
__device__ __forceinline__ uint32_t quantise(float p, double step, float lo, float hi) {
    double ql = floor(((double)lo - (double)p) / step - 0x1p-20);
    double qh = ceil(((double)hi - (double)p) / step + 0x1p-20);
    ql = fmin(fmax(ql, 0.0), 65535.0);
    qh = fmin(fmax(qh, 0.0), 65535.0);
    return (uint32_t)ql | ((uint32_t)qh << 16);
}

// ctrs[0]: items of the next level, [1]: nodes allocated, [2]: error, [3]: triangles placed
__global__ void k_collapse(const float4 *__restrict__ bin, uint32_t n_records, const CollapseItem *__restrict__ in,
                           uint32_t n_in, CollapseItem *out, uint32_t cap, uint4 *nodes, const float4 *__restrict__ mtris,
                           float4 *tris, uint32_t n_tri, uint32_t *ctrs) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_in) return;
    const CollapseItem it = in[i];
    uint32_t rec[kWide];
    int m = (int)it.seeds;
    rec[0] = it.rec;
    rec[1] = it.rec + 1u;
    if ((uint64_t)it.rec + (uint64_t)it.seeds > n_records || it.node >= cap) { atomicMax(&ctrs[2], 1u); return; }
    for (;;) {   // open the internal child with the largest box while there is room
        if (m >= kWide) break;
        int best = -1;
        float best_area = -1.0f;
        for (int k = 0; k < m; ++k) {
            if (!rec_internal(bin, rec[k])) continue;
            const float a = half_area(bin[2 * (size_t)rec[k]], bin[2 * (size_t)rec[k] + 1]);
            if (a > best_area) { best_area = a; best = k; }
        }
        if (best < 0) break;
        const uint32_t a = __float_as_uint(bin[2 * (size_t)rec[best]].w);
        if (a < 2u || (uint64_t)a + 1u >= n_records) { atomicMax(&ctrs[2], 1u); return; }
        rec[best] = a;
        rec[m++] = a + 1u;
    }
    float4 lo[kWide], hi[kWide];
    float4 nlo = make_float4(3.0e38f, 3.0e38f, 3.0e38f, 0.0f), nhi = make_float4(-3.0e38f, -3.0e38f, -3.0e38f, 0.0f);
    for (int k = 0; k < m; ++k) {
        lo[k] = bin[2 * (size_t)rec[k]];
        hi[k] = bin[2 * (size_t)rec[k] + 1];
        nlo = make_float4(fminf(nlo.x, lo[k].x), fminf(nlo.y, lo[k].y), fminf(nlo.z, lo[k].z), 0.0f);
        nhi = make_float4(fmaxf(nhi.x, hi[k].x), fmaxf(nhi.y, hi[k].y), fmaxf(nhi.z, hi[k].z), 0.0f);
    }
    // (keeping the internal children of a full node that hold at most 3 triangles as leaves instead:
    // 38 % fewer nodes on the 1,000,000-triangle soup, 4.5x the triangle tests, 1.3 % slower)
    bool internal[kWide];
    for (int k = 0; k < m; ++k) internal[k] = rec_internal(bin, rec[k]);
    // slots by octant: the child whose centre lies on the high side of axis a prefers slots with bit a set
    const float cx = 0.5f * (nlo.x + nhi.x), cy = 0.5f * (nlo.y + nhi.y), cz = 0.5f * (nlo.z + nhi.z);
    int slot_of[kWide];
    uint32_t used = 0, placed = 0;
    for (int k = 0; k < m; ++k) slot_of[k] = -1;
    for (int round = 0; round < m; ++round) {
        float best = 3.0e38f;
        int bk = -1, bs = -1;
        for (int k = 0; k < m; ++k) {
            if ((placed >> k) & 1u) continue;
            const float dx = 0.5f * (lo[k].x + hi[k].x) - cx, dy = 0.5f * (lo[k].y + hi[k].y) - cy,
                        dz = 0.5f * (lo[k].z + hi[k].z) - cz;
            for (int sl = 0; sl < kWide; ++sl) {
                if ((used >> sl) & 1u) continue;
                const float c = ((sl & 1) ? -dx : dx) + ((sl & 2) ? -dy : dy) + ((sl & 4) ? -dz : dz);
                if (c < best) { best = c; bk = k; bs = sl; }
            }
        }
        if (bk < 0) {   // non-finite centres: the first free slot
            bk = __ffs(~placed & ((1u << m) - 1u)) - 1;
            bs = __ffs(~used & 0xFFu) - 1;
        }
        slot_of[bk] = bs;
        placed |= 1u << bk;
        used |= 1u << bs;
    }
    int child_at[kWide];
    for (int sl = 0; sl < kWide; ++sl) child_at[sl] = -1;
    uint32_t imask = 0, n_int = 0, n_lt = 0;
    for (int k = 0; k < m; ++k) {
        child_at[slot_of[k]] = k;
        if (internal[k]) { imask |= 1u << slot_of[k]; ++n_int; }
        else n_lt += (uint32_t)__float_as_int(hi[k].w);
    }
    const uint32_t child_base = n_int ? atomicAdd(&ctrs[1], n_int) : 0u;
    const uint32_t qpos = n_int ? atomicAdd(&ctrs[0], n_int) : 0u;
    const uint32_t tri_base = n_lt ? atomicAdd(&ctrs[3], n_lt) : 0u;
    if ((uint64_t)child_base + n_int > cap || (uint64_t)qpos + n_int > cap || (uint64_t)tri_base + n_lt > n_tri) {
        atomicMax(&ctrs[2], 1u);
        return;
    }
    const int ex = grid_exponent(nlo.x, nhi.x), ey = grid_exponent(nlo.y, nhi.y), ez = grid_exponent(nlo.z, nhi.z);
    if (ex > 127 || ey > 127 || ez > 127) { atomicMax(&ctrs[2], 2u); return; }
    const double sx = ldexp(1.0, ex), sy = ldexp(1.0, ey), sz = ldexp(1.0, ez);
    uint32_t w[kNodeWords];
    w[0] = __float_as_uint(nlo.x);
    w[1] = __float_as_uint(nlo.y);
    w[2] = __float_as_uint(nlo.z);
    w[3] = (uint32_t)(ex + 127) | ((uint32_t)(ey + 127) << 8) | ((uint32_t)(ez + 127) << 16) | (imask << 24);
    w[kNodeChildBase] = child_base;
    w[kNodeTriBase] = tri_base;
    w[kNodeMeta] = w[kNodeMeta + 1] = 0;
    uint32_t offset = 0, rank = 0;
    for (int sl = 0; sl < kWide; ++sl) {
        const int k = child_at[sl];
        if (k < 0) {   // empty slot: an inverted box, no meta
            w[node_plane_word(0, sl)] = w[node_plane_word(1, sl)] = w[node_plane_word(2, sl)] = 0xFFFFu;
            continue;
        }
        w[node_plane_word(0, sl)] = quantise(nlo.x, sx, lo[k].x, hi[k].x);
        w[node_plane_word(1, sl)] = quantise(nlo.y, sy, lo[k].y, hi[k].y);
        w[node_plane_word(2, sl)] = quantise(nlo.z, sz, lo[k].z, hi[k].z);
        if ((imask >> sl) & 1u) {
            out[qpos + rank] = CollapseItem{__float_as_uint(lo[k].w), 2u, child_base + rank};
            ++rank;
        } else {
            const uint32_t first = __float_as_uint(lo[k].w), count = (uint32_t)__float_as_int(hi[k].w);
            if (count == 0 || count > kMaxLeafTris || (uint64_t)first + count > n_tri) { atomicMax(&ctrs[2], 1u); return; }
            w[kNodeMeta + (sl >> 2)] |= ((((1u << count) - 1u) << 5) | offset) << (8 * (sl & 3));
            for (uint32_t j = 0; j < count; ++j)
                for (int c = 0; c < 3; ++c) tris[3 * (size_t)(tri_base + offset + j) + c] = mtris[3 * (size_t)(first + j) + c];
            offset += count;
        }
    }
    uint4 *dst = nodes + (size_t)it.node * (kNodeWords / 4);
    for (int q = 0; q < kNodeWords / 4; ++q) dst[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
}

}  // namespace

namespace mrt_host {

int leaf_max_setting() {
    static int v = [] {
        const char *e = getenv("MRT_BVH_LEAF_MAX");
        const int x = e ? atoi(e) : (int)kMaxLeafTris;   // the largest subtree the surface-area leaf choice may keep as one leaf
        return x < 1 ? 1 : (x > (int)kMaxLeafTris ? (int)kMaxLeafTris : x);
    }();
    return v;
}

int build_fast_bvh(MrtScene *s) {
    MrtContext *ctx = s->ctx;
    cudaStream_t q = ctx->stream;
    const uint32_t n = s->n_tri;
    // planes and spheres are walked in order in FAST mode; only triangles get the tree
    if (n == 0) {
        s->fnode_count = 0;
        s->dev.n_fnodes = 0;
        s->dev.fnodes = nullptr;
        s->dev.ftris = nullptr;
        return MRT_OK;
    }
    if (n >= kMaxFastTris) {
        set_error(ctx, "fast bvh: at most %u triangles", kMaxFastTris - 1u);
        return MRT_ERR_ARG;
    }
    int st = MRT_OK;
    const uint64_t n_records = 2ull + 2ull * (n > 1 ? n - 1 : 0) + 2ull;
    st = dev_alloc(ctx, s->fnodes, 32ull * n_records);
    if (st == MRT_OK) st = dev_alloc(ctx, s->ftris, 48ull * n);
    if (st != MRT_OK) return st;
    DevBuf bmin, bmax, cb, keys[2], vals[2], hist, lft, rgt, fst, lst, pint, pleaf, ctr, imin, imax, mtris;
    const uint32_t nblocks = (n + kSortTile - 1) / kSortTile;
    auto A = [&](DevBuf &b, size_t bytes) { if (st == MRT_OK) st = dev_alloc(ctx, b, bytes); };
    A(bmin, 16ull * n); A(bmax, 16ull * n); A(cb, 64);
    A(keys[0], 4ull * n); A(keys[1], 4ull * n); A(vals[0], 4ull * n); A(vals[1], 4ull * n);
    A(hist, 4ull * 256 * nblocks);
    A(lft, 4ull * n); A(rgt, 4ull * n); A(fst, 4ull * n); A(lst, 4ull * n);
    A(pint, 4ull * n); A(pleaf, 4ull * n); A(ctr, 4ull * n); A(imin, 16ull * n); A(imax, 16ull * n);
    A(mtris, 48ull * n);
    if (st == MRT_OK) {
        const uint32_t init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
        st = cuda_status(ctx, cudaMemcpyAsync(cb.ptr, init, sizeof(init), cudaMemcpyHostToDevice, q), "bvh init");
    }
    if (st == MRT_OK) {
        const uint32_t g = (n + 255) / 256;
        k_tri_boxes<<<g, 256, 0, q>>>(n, s->dev.tri_a, s->dev.tri_ab, s->dev.tri_ac, (float4 *)bmin.ptr,
                                      (float4 *)bmax.ptr, (uint32_t *)cb.ptr);
        k_morton<<<g, 256, 0, q>>>(n, (const float4 *)bmin.ptr, (const float4 *)bmax.ptr, (const uint32_t *)cb.ptr,
                                   (uint32_t *)keys[0].ptr, (uint32_t *)vals[0].ptr);
        int cur = 0;
        for (int shift = 0; shift < 30; shift += 8) {
            k_rs_hist<<<nblocks, kSortThreads, 0, q>>>((const uint32_t *)keys[cur].ptr, n, shift, (uint32_t *)hist.ptr, nblocks);
            k_scan_exclusive<<<1, 1024, 0, q>>>((uint32_t *)hist.ptr, 256u * nblocks);
            k_rs_scatter<<<nblocks, kSortThreads, 0, q>>>((const uint32_t *)keys[cur].ptr, (const uint32_t *)vals[cur].ptr,
                                                          (uint32_t *)keys[1 - cur].ptr, (uint32_t *)vals[1 - cur].ptr, n,
                                                          shift, (const uint32_t *)hist.ptr, nblocks);
            cur = 1 - cur;
        }
        const uint32_t *skeys = (const uint32_t *)keys[cur].ptr;
        const uint32_t *svals = (const uint32_t *)vals[cur].ptr;
        if (n == 1) {
            k_single_leaf<<<1, 1, 0, q>>>((const float4 *)bmin.ptr, (const float4 *)bmax.ptr, (float4 *)s->fnodes.ptr);
        } else {
            cudaMemsetAsync(ctr.ptr, 0, 4ull * n, q);
            k_karras<<<(n - 1 + 255) / 256, 256, 0, q>>>((int)n, skeys, (uint32_t *)lft.ptr, (uint32_t *)rgt.ptr,
                                                          (uint32_t *)fst.ptr, (uint32_t *)lst.ptr, (uint32_t *)pint.ptr,
                                                          (uint32_t *)pleaf.ptr);
            k_fit<<<(n + 255) / 256, 256, 0, q>>>((int)n, svals, (const float4 *)bmin.ptr, (const float4 *)bmax.ptr,
                                                  (const uint32_t *)lft.ptr, (const uint32_t *)rgt.ptr,
                                                  (const uint32_t *)pint.ptr, (const uint32_t *)pleaf.ptr,
                                                  (uint32_t *)ctr.ptr, (float4 *)imin.ptr, (float4 *)imax.ptr);
            k_emit<<<(n - 1 + 255) / 256, 256, 0, q>>>((int)n, leaf_max_setting(), svals, (const float4 *)bmin.ptr,
                                                       (const float4 *)bmax.ptr, (const uint32_t *)lft.ptr,
                                                       (const uint32_t *)rgt.ptr, (const uint32_t *)fst.ptr,
                                                       (const uint32_t *)lst.ptr, (const float4 *)imin.ptr,
                                                       (const float4 *)imax.ptr, (float4 *)s->fnodes.ptr);
        }
        k_leaf_tris<<<(n + 255) / 256, 256, 0, q>>>(n, svals, s->dev.tri_a, s->dev.tri_ab, s->dev.tri_ac,
                                                    (float4 *)mtris.ptr);
        st = cuda_status(ctx, cudaGetLastError(), "fast bvh kernels");
        if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "fast bvh build");
    }
    DevBuf *tmp[] = {&bmin, &bmax, &cb, &keys[0], &keys[1], &vals[0], &vals[1], &hist, &lft, &rgt, &fst, &lst,
                     &pint, &pleaf, &ctr, &imin, &imax};
    for (DevBuf *b : tmp) dev_free(*b);
    if (st != MRT_OK) { dev_free(mtris); return st; }
    // collapse into 8-wide compressed nodes, level by level, from the root record
    DevBuf wide, queue[2], wctr;
    const uint32_t cap = n;   // wide nodes <= binary internal nodes + 1
    A(wide, 4ull * kNodeWords * cap);
    A(queue[0], sizeof(CollapseItem) * cap);
    A(queue[1], sizeof(CollapseItem) * cap);
    A(wctr, 16);
    uint32_t h[4] = {1, 1, 0, 0};   // the root item, the root node
    if (st == MRT_OK) {
        const CollapseItem root{0u, 1u, 0u};
        st = cuda_status(ctx, cudaMemcpyAsync(queue[0].ptr, &root, sizeof(root), cudaMemcpyHostToDevice, q), "collapse");
        if (st == MRT_OK) st = cuda_status(ctx, cudaMemcpyAsync(wctr.ptr, h, 16, cudaMemcpyHostToDevice, q), "collapse");
    }
    int cur_q = 0;
    for (int level = 0; st == MRT_OK && h[0] > 0 && h[2] == 0; ++level) {
        if (level > 4096) { st = MRT_ERR_LIMIT; break; }
        const uint32_t n_in = h[0];
        cudaMemsetAsync(wctr.ptr, 0, 4, q);
        k_collapse<<<(n_in + 127) / 128, 128, 0, q>>>((const float4 *)s->fnodes.ptr, (uint32_t)n_records,
                                                       (const CollapseItem *)queue[cur_q].ptr, n_in,
                                                       (CollapseItem *)queue[1 - cur_q].ptr, cap, (uint4 *)wide.ptr,
                                                       (const float4 *)mtris.ptr, (float4 *)s->ftris.ptr, n,
                                                       (uint32_t *)wctr.ptr);
        cur_q = 1 - cur_q;
        st = cuda_status(ctx, cudaMemcpyAsync(h, wctr.ptr, 16, cudaMemcpyDeviceToHost, q), "collapse");
        if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "collapse");
    }
    if (st == MRT_OK && (h[2] != 0 || h[3] != n)) {
        set_error(ctx, h[2] == 2 ? "fast bvh: scene extent beyond the 2^127 grid step"
                                 : "fast bvh: inconsistent binary tree while collapsing");
        st = MRT_ERR_LIMIT;
    }
    const uint64_t n_wide = h[1];
    if (st == MRT_OK) {   // exact-size copy; the binary records and the scratch go
        dev_free(s->fnodes);
        st = dev_alloc(ctx, s->fnodes, 4ull * kNodeWords * n_wide);
        if (st == MRT_OK)
            st = cuda_status(ctx, cudaMemcpyAsync(s->fnodes.ptr, wide.ptr, 4ull * kNodeWords * n_wide,
                                                  cudaMemcpyDeviceToDevice, q), "collapse copy");
        if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "collapse copy");
    }
    DevBuf *tmp2[] = {&wide, &queue[0], &queue[1], &wctr, &mtris};
    for (DevBuf *b : tmp2) dev_free(*b);
    if (st != MRT_OK) return st;
    s->fnode_count = n_wide;
    s->dev.n_fnodes = (uint32_t)n_wide;
    s->dev.fnodes = (const float4 *)s->fnodes.ptr;
    s->dev.ftris = (const float4 *)s->ftris.ptr;
    return MRT_OK;
}

int build_reference_bvh(MrtScene *s) {
    MrtContext *ctx = s->ctx;
    for (int k = 0; k < 3; ++k) {
        std::vector<HBox> boxes;
        if (k == kTriangle) {
            boxes.resize(s->n_tri);
            for (uint32_t i = 0; i < s->n_tri; ++i) {   // Triangle::getAABB, Triangle.cpp:145-152
                const float *p = &s->h_abc[9ull * i];
                const V3 A{p[0], p[1], p[2]};
                const V3 ab = V3{p[3], p[4], p[5]} - A, ac = V3{p[6], p[7], p[8]} - A;
                const V3 B = A + ab, C = A + ac;
                boxes[i] = HBox{vmin(A, vmin(B, C)), vmax(A, vmax(B, C))};
            }
        } else if (k == kSphere) {
            boxes.resize(s->n_sph);
            for (uint32_t i = 0; i < s->n_sph; ++i) {   // Sphere::getAABB, Sphere.cpp:94-100
                const float *c = &s->h_sph[4ull * i];
                const float r = sqrtf(c[3]);
                const V3 ctr{c[0], c[1], c[2]};
                boxes[i] = HBox{subs(ctr, r), adds(ctr, r)};
            }
        } else {
            boxes.resize(s->n_pln);
            for (uint32_t i = 0; i < s->n_pln; ++i) {   // Plane::getAABB / getRightVector, Plane.cpp:80-105
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
                boxes[i] = HBox{pt + right * -100.0f, pt + right * 100.0f};
            }
        }
        const std::vector<RefNode> nodes = ref_build(boxes);
        int st = dev_alloc(ctx, s->rnodes[k], sizeof(RefNode) * nodes.size());
        if (st == MRT_OK)
            st = cuda_status(ctx, cudaMemcpyAsync(s->rnodes[k].ptr, nodes.data(), sizeof(RefNode) * nodes.size(),
                                                  cudaMemcpyHostToDevice, ctx->stream), "upload bvh");
        if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "upload bvh");
        if (st != MRT_OK) return st;
        s->rnode_count[k] = nodes.size();
        s->dev.rnodes[k] = (const RefNode *)s->rnodes[k].ptr;
        s->dev.rnode_count[k] = (uint32_t)nodes.size();
    }
    return MRT_OK;
}

}  // namespace mrt_host
