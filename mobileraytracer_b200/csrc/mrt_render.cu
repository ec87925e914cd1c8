// mrt_render.cu - Renderer::renderFrame on the device (Renderer.cpp:31-116).
//
// Pixels: the reference renders 16x16 blocks handed out in a shuffled Halton order
// (Camera.cpp:13-37, Renderer.cpp:79-93); each visited pixel gets, per sample pass,
// bitmap = incrementalAvg(rgb, bitmap, sample + 1).  The host enumerates the visited pixels with the
// reference's block arithmetic; when they form the rectangle [0,W) x [0,16*(H/16)) with no pixel
// visited twice (the usual case) the kernels map threads to pixels directly, otherwise they walk an
// explicit task list in block order, one round per repeated visit.
//
// NoShadows (NoShadows.cpp:19-65) has no secondary rays: one fused kernel does camera ray, closest
// hit, shading and the running mean per pixel.
//
// Whitted and PathTracer (Whitted.cpp:17-107, PathTracer.cpp:25-164) recurse.  Here they run as a
// wavefront over a wave of camera paths: per bounce level an extend kernel (closest hit), a shade
// kernel that writes one node record per ray and appends shadow rays and continuation rays to
// queues compacted with warp ballots, and an any-hit kernel for the shadow queue.  After the last
// level the nodes are resolved bottom-up, level by level, combining each node's own terms with its
// children's results in the reference's order of operations, so the per-sample value equals the
// recursive one bit for bit.  Per-sample values are then folded into the bitmap in sample order.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>

#include "mrt_gridwalk.cuh"
#include "mrt_internal.h"
#include "mrt_paths.cuh"

using namespace mrt;
using namespace mrt_host;

namespace {

template <int ACCEL, int MODE>
__global__ void __launch_bounds__(128) k_render_noshadows(DevScene s, RenderParams p, uint32_t round_first,
                                                          uint32_t round_count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < round_count; i += gridDim.x * blockDim.x) {
        const uint32_t t = round_first + i;
        const Task k = task_of(p, t);
        const uint32_t pixel = k.y * p.width + k.x;
        const int64_t slot = p.accum ? accum_slot(p, k) : -1;
        uint32_t bm = p.bitmap[k.index];
        float4 acc = slot >= 0 ? p.accum[slot] : make_float4(0, 0, 0, 0);
        for (uint32_t si = 0; si < p.spp; ++si) {
            const uint32_t sample = p.spp_offset + si;
            const Stream st = make_stream(p.seed, pixel, sample, p.strata, p.constant_value);
            const Ray r = primary_ray(p, k, st);
            V3 rgb{0.0f, 0.0f, 0.0f};
            float len;
            uint32_t id;
            if (scene_closest<ACCEL, MODE>(s, r, len, id)) {
                Isect it;
                if (make_isect(s, r, id, it)) rgb = shade_direct(s, p, st, r, it);
            }
            bm = incremental_avg(rgb, bm, sample + 1u);
            acc.x += rgb.x; acc.y += rgb.y; acc.z += rgb.z; acc.w += 1.0f;
        }
        p.bitmap[k.index] = bm;
        if (slot >= 0) p.accum[slot] = acc;
    }
}


// persistent FAST-BVH NoShadows: work item = pixel task; the lane traces the pixel's samples in
// order.  Only the task number and the sample count stay in registers while a ray is traced: the
// pixel's running mean and fp32 sums are read and written back at the end of each sample (a few
// bytes per ray), which leaves the registers to the traversal.  Implicit tasks are fetched in
// 2x16-pixel tiles (when the image allows) so the rays of a warp start coherent; tiles are handed
// out row by row.  On the 1,000,000-triangle soup frame 2x16 tiles beat 4x8 by 0.7 % and 8x4 by
// 3.3 %; handing out 64x32-pixel regions per SM, or the tiles in vertical strips, was slower.
struct NsLane {
    uint32_t t;    // task number
    uint32_t si;   // samples done
};

// task of the round's item-th pixel: row-major from `first`, or in 2x16-pixel tiles handed out row
// by row (tiles_x tiles per tile row)
__device__ __forceinline__ uint32_t ns_task(const RenderParams &p, uint32_t first, uint32_t item, uint32_t tiles_x) {
    if (!tiles_x) return first + item;
    const uint32_t tile = item >> 5, w = item & 31u;
    const uint32_t x = (tile % tiles_x) * 2u + (w & 1u), y = (tile / tiles_x) * 16u + (w >> 1);
    return y * p.width + x;
}

struct NsWork {
    const DevScene *s;
    const RenderParams *p;
    uint32_t first, count;
    uint32_t *ctr;
    uint32_t tiles_x;   // tiles per tile row (0: row-major tasks)
    __device__ uint32_t total() const { return count; }
    __device__ uint32_t *counter() const { return ctr; }
    template <class L>
    __device__ const DevScene &scene(const L &, const DevScene &s) const { return s; }
    template <class L>
    __device__ const DevScene &view(const L &, const DevScene &s) const { return s; }
    __device__ Ray ray_for(const NsLane &lane) const {
        const Task k = task_of(*p, lane.t);
        const Stream st = make_stream(p->seed, k.y * p->width + k.x, p->spp_offset + lane.si, p->strata, p->constant_value);
        return primary_ray(*p, k, st);
    }
    __device__ bool begin(uint32_t item, NsLane &lane, Ray &r) const {
        lane.t = ns_task(*p, first, item, tiles_x);
        lane.si = 0;
        r = ray_for(lane);
        return true;
    }
    __device__ bool finish(NsLane &lane, Ray &r, bool hit, float, uint32_t id, const FastTrav &) const {
        const Task k = task_of(*p, lane.t);
        const uint32_t sample = p->spp_offset + lane.si;
        V3 rgb{0.0f, 0.0f, 0.0f};
        if (hit) {
            Isect it;
            if (make_isect(*s, r, id, it)) {
                const Stream st = make_stream(p->seed, k.y * p->width + k.x, sample, p->strata, p->constant_value);
                rgb = shade_direct(*s, *p, st, r, it);
            }
        }
        p->bitmap[k.index] = incremental_avg(rgb, p->bitmap[k.index], sample + 1u);
        const int64_t slot = p->accum ? accum_slot(*p, k) : -1;
        if (slot >= 0) {
            float4 acc = p->accum[slot];
            acc.x += rgb.x; acc.y += rgb.y; acc.z += rgb.z; acc.w += 1.0f;
            p->accum[slot] = acc;
        }
        if (++lane.si < p->spp) {
            r = ray_for(lane);
            return true;
        }
        return false;
    }
};

// resident blocks of 128 threads per SM for the NoShadows traversal (registers per thread: 65536 / (128 x
// this)).  On the 1,000,000-triangle soup frame the split trace kernel fits 72 registers without spills:
// 7 blocks give 1507 Mrays/s against 1454 at 6 (80 registers) and 1353 at 8 (64 registers, spills).
#ifndef MRT_NS_BLOCKS_PER_SM
#define MRT_NS_BLOCKS_PER_SM 7
#endif
constexpr int kNsBlocksPerSm = MRT_NS_BLOCKS_PER_SM;

__global__ void __launch_bounds__(128, kNsBlocksPerSm) k_render_noshadows_fast(DevScene s, RenderParams p, uint32_t first,
                                                               uint32_t count, uint32_t *ctr, uint32_t tiles_x) {
    NsWork w{&s, &p, first, count, ctr, tiles_x};
    NsLane lane;
    persistent_closest<false>(s, w, lane);
}

// the same work on the RegularGrid: the persistent grid walk (mrt_gridwalk.cuh), one cell per lane
// and loop iteration
__global__ void __launch_bounds__(128, kGridBlocksPerSm) k_render_noshadows_grid(DevScene s, RenderParams p, uint32_t first,
                                                               uint32_t count, uint32_t *ctr, uint32_t tiles_x) {
    NsWork w{&s, &p, first, count, ctr, tiles_x};
    NsLane lane;
    persistent_grid_closest(s, w, lane);
}

// NoShadows on the FAST tree in two passes over a chunk of (sample, pixel) items: the persistent
// traversal writes each camera ray's closest hit (distance bits, hit id) to a buffer, then one
// thread per pixel shades the chunk's samples in sample order and updates the running mean.  The
// traversal lanes then carry nothing but their item (no shading code between node steps: fewer
// registers, and the shading runs with every lane of a warp busy instead of the few lanes that
// finish a ray in the same iteration).
struct NsTraceLane {
    uint32_t i;   // item of the chunk
};

struct NsTraceWork {
    const RenderParams *p;
    uint32_t first, j0, n_pix, s0, n_items, tiles_x;
    uint32_t *ctr;
    uint2 *hits;
    __device__ uint32_t total() const { return n_items; }
    __device__ uint32_t *counter() const { return ctr; }
    template <class L>
    __device__ const DevScene &scene(const L &, const DevScene &s) const { return s; }
    template <class L>
    __device__ const DevScene &view(const L &, const DevScene &s) const { return s; }
    __device__ bool begin(uint32_t item, NsTraceLane &lane, Ray &r) const {
        lane.i = item;
        const uint32_t si = item / n_pix, j = item - si * n_pix;
        const Task k = task_of(*p, ns_task(*p, first, j0 + j, tiles_x));
        const Stream st = make_stream(p->seed, k.y * p->width + k.x, p->spp_offset + s0 + si, p->strata, p->constant_value);
        r = primary_ray(*p, k, st);
        return true;
    }
    __device__ bool finish(NsTraceLane &lane, Ray &, bool hit, float t, uint32_t id, const FastTrav &) const {
        hits[lane.i] = make_uint2(__float_as_uint(t), hit ? id : MRT_HIT_NONE);
        return false;
    }
};

// the split form (0: one fused kernel traces and shades) and its chunk of items (hit buffer of 8 B each)
#ifndef MRT_NS_SPLIT
#define MRT_NS_SPLIT 1
#endif
constexpr bool kNsSplit = MRT_NS_SPLIT != 0;
// host-memory frames shaded in bands whose copies out overlap the shading (0: one copy at the end)
#ifndef MRT_HOST_BANDS
#define MRT_HOST_BANDS 1
#endif
constexpr bool kHostBandsOn = MRT_HOST_BANDS != 0;
// node-phase quorum of the NoShadows traversal (coherent camera rays)
constexpr int kNsQuorum = kCameraQuorum;
// idle lanes that trigger a refill in the NoShadows traversal
#ifndef MRT_NS_REFILL
#define MRT_NS_REFILL 8
#endif
constexpr int kNsRefill = MRT_NS_REFILL;
constexpr uint32_t kNsChunk = 1u << 22;

__global__ void __launch_bounds__(128, kNsBlocksPerSm) k_ns_trace(DevScene s, NsTraceWork w, RenderParams p) {
    w.p = &p;
    NsTraceLane lane;
    // (the first 8, 16 or 32 stack entries in shared memory instead of local memory: 2-6 % slower)
    persistent_closest<false, kNsQuorum, kNsRefill>(s, w, lane);
}

// the same traversal pass on the RegularGrid (the persistent grid walk)
__global__ void __launch_bounds__(128, kGridBlocksPerSm) k_ns_trace_grid(DevScene s, NsTraceWork w, RenderParams p) {
    w.p = &p;
    NsTraceLane lane;
    persistent_grid_closest(s, w, lane);
}

// shading of items j0 .. j0 + n_pix - 1 of a traced chunk: the hit of sample si of item j0 + j is
// hits[si * hit_stride + j] (hit_stride = the chunk's item count; a band of the chunk passes the hits
// from its first item on)
__global__ void __launch_bounds__(128) k_ns_shade(DevScene s, RenderParams p, uint32_t first, uint32_t j0, uint32_t n_pix,
                                                  uint32_t s0, uint32_t n_s, uint32_t tiles_x, const uint2 *__restrict__ hits,
                                                  uint32_t hit_stride) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n_pix; j += gridDim.x * blockDim.x) {
        const Task k = task_of(p, ns_task(p, first, j0 + j, tiles_x));
        uint32_t bm = p.bitmap[k.index];
        const int64_t slot = p.accum ? accum_slot(p, k) : -1;
        float4 acc = slot >= 0 ? p.accum[slot] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (uint32_t si = 0; si < n_s; ++si) {
            const uint32_t sample = p.spp_offset + s0 + si;
            const uint2 h = hits[(size_t)si * hit_stride + j];
            V3 rgb{0.0f, 0.0f, 0.0f};
            if (h.y != MRT_HIT_NONE) {
                const Stream st = make_stream(p.seed, k.y * p.width + k.x, sample, p.strata, p.constant_value);
                const Ray r = primary_ray(p, k, st);
                Isect it;
                if (make_isect(s, r, h.y, it)) rgb = shade_direct(s, p, st, r, it);
            }
            bm = incremental_avg(rgb, bm, sample + 1u);
            acc.x += rgb.x; acc.y += rgb.y; acc.z += rgb.z; acc.w += 1.0f;
        }
        p.bitmap[k.index] = bm;
        if (slot >= 0) p.accum[slot] = acc;
    }
}

// ============================== wavefront ====================================================
__global__ void k_wave_raygen(RenderParams p, WaveState w) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < w.n_roots; i += gridDim.x * blockDim.x) {
        Task k;
        uint32_t pixel, sample;
        root_task(p, w, i, k, pixel, sample);
        const Stream st = make_stream(p.seed, pixel, sample, p.strata, p.constant_value);
        const Ray r = primary_ray(p, k, st);
        RayRec rr;
        rr.ox = r.o.x; rr.oy = r.o.y; rr.oz = r.o.z;
        rr.dx = r.d.x; rr.dy = r.d.y; rr.dz = r.d.z;
        rr.depth = 1;
        rr.exclude = MRT_HIT_NONE;
        rr.root = i;
        rr.parent = 0xFFFFFFFFu;
        rr.slot = 0;
        rr.code = 1u;
        w.rays[i] = rr;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.levels[0].start = 0;
        w.levels[0].count = w.n_roots;
        w.levels[0].shadow_count = 0;
    }
}
template <int ACCEL, int MODE>
__global__ void __launch_bounds__(128) k_wave_extend(DevScene s, WaveState w, int level) {
    const Level L = clamp_level(w, w.levels[level]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.count; i += gridDim.x * blockDim.x) {
        const uint32_t idx = L.start + i;
        const Ray r = ray_of(w.rays[idx]);
        float len;
        uint32_t id;
        const bool hit = scene_closest<ACCEL, MODE>(s, r, len, id);
        w.nodes[idx].hit_t = len;
        w.nodes[idx].hit_id = hit ? id : MRT_HIT_NONE;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&w.counters[0], (unsigned long long)L.count);
}

// one ray of a level shaded; every lane of the warp calls this (the child and shadow queues are
// allocated once per warp)
__device__ __forceinline__ void shade_slot(const DevScene &s, const RenderParams &p, const WaveState &w, int level,
                                           Level *next, uint32_t next_start, bool active, uint32_t idx) {
    ShadeLane o;
    o.n_child = 0;
    o.child_mask = 0;
    o.n_shadow = 0;
    o.shaded = false;
    RayRec rr;
    Stream st;
    if (active) {
        rr = w.rays[idx];
        Task k;
        uint32_t pixel, sample;
        root_task(p, w, rr.root, k, pixel, sample);
        st = make_stream(p.seed, pixel, sample, p.strata, p.constant_value);
        shade_ray(s, p, rr, w.nodes[idx].hit_id, w.nodes[idx].hit_t, st, o);
        store_node(w.nodes[idx], o.nd);
    }
    // queue compaction: one atomic per warp for children, one for shadow rays
    const uint32_t cbase = warp_alloc(o.n_child, &next->count);
    const uint32_t sbase = warp_alloc(o.n_shadow, &w.levels[level].shadow_count);
    if (!active) return;
    emit_children(s, o, rr, st, idx, next_start + cbase, w.rays, w.ray_cap);
    emit_shadows(s, p, st, o, rr, idx, sbase, w.shadows, w.shadow_cap);
}

__global__ void __launch_bounds__(128) k_wave_shade(DevScene s, RenderParams p, WaveState w, int level) {
    const Level L = clamp_level(w, w.levels[level]);
    Level *next = &w.levels[level + 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) next->start = L.start + L.count;
    const uint32_t next_start = L.start + L.count;
    const uint32_t n_iter = (L.count + blockDim.x - 1) / blockDim.x;   // whole warps iterate together
    for (uint32_t it_ = blockIdx.x; it_ < n_iter; it_ += gridDim.x) {
        const uint32_t i = it_ * blockDim.x + threadIdx.x;
        const bool active = i < L.count;
        shade_slot(s, p, w, level, next, next_start, active, L.start + (active ? i : 0u));
    }
}

// Per-material shade queues for scenes that mix diffuse with mirror / glass materials: a block takes
// a window of kSortRounds x 128 consecutive rays of the level, sorts them by shading class in shared
// memory (one warp ballot per class and round; the class sizes by shared-memory atomics of the
// ballots' popc, then each ray's place = its class's offset + its warp's share + its rank among the
// ballot's lanes) and shades the window in that order, so that all but at most two warps of a
// window run one material branch.  The reordered reads stay within the window's 180 KB of ray and
// node records, most of them in L1 or L2 (a global sort of the level scatters every record access,
// and its extra pass cost more than the divergence it removed).
constexpr int kSortRounds = 8;
__global__ void __launch_bounds__(128) k_wave_shade_sorted(DevScene s, RenderParams p, WaveState w, int level) {
    __shared__ uint32_t s_idx[kSortRounds * 128];
    __shared__ uint32_t s_cnt[kShadeClasses], s_fill[kShadeClasses];
    const Level L = clamp_level(w, w.levels[level]);
    Level *next = &w.levels[level + 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) next->start = L.start + L.count;
    const uint32_t next_start = L.start + L.count;
    const uint32_t win = kSortRounds * 128u;
    const uint32_t n_win = (L.count + win - 1) / win;
    const uint32_t FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const uint32_t lanes_below = (1u << lane) - 1u;
    for (uint32_t wi = blockIdx.x; wi < n_win; wi += gridDim.x) {
        const uint32_t base = wi * win;
        const uint32_t n_here = min(win, L.count - base);
        if (threadIdx.x < kShadeClasses) {
            s_cnt[threadIdx.x] = 0;
            s_fill[threadIdx.x] = 0;
        }
        __syncthreads();
        uint32_t classes = 0;   // 2 bits per round; 3 = no ray
#pragma unroll
        for (int r = 0; r < kSortRounds; ++r) {
            const uint32_t j = r * 128u + threadIdx.x;
            const uint32_t idx = L.start + base + j;
            const uint32_t c = j < n_here ? shade_class(s, p, w.rays[idx], w.nodes[idx].hit_id) : 3u;
            classes |= c << (2 * r);
#pragma unroll
            for (uint32_t k = 0; k < (uint32_t)kShadeClasses; ++k) {
                const uint32_t m = __ballot_sync(FULL, c == k);
                if (lane == 0 && m) atomicAdd(&s_cnt[k], (uint32_t)__popc(m));
            }
        }
        __syncthreads();
        const uint32_t off[kShadeClasses] = {0u, s_cnt[0], s_cnt[0] + s_cnt[1]};
#pragma unroll
        for (int r = 0; r < kSortRounds; ++r) {
            const uint32_t c = (classes >> (2 * r)) & 3u;
#pragma unroll
            for (uint32_t k = 0; k < (uint32_t)kShadeClasses; ++k) {
                const uint32_t m = __ballot_sync(FULL, c == k);
                if (!m) continue;
                const int leader = __ffs(m) - 1;
                uint32_t b = 0;
                if (lane == leader) b = atomicAdd(&s_fill[k], (uint32_t)__popc(m));
                b = __shfl_sync(FULL, b, leader);
                if (c == k) s_idx[off[k] + b + __popc(m & lanes_below)] = base + r * 128u + threadIdx.x;
            }
        }
        __syncthreads();
        for (int r = 0; r < kSortRounds; ++r) {
            const uint32_t j = r * 128u + threadIdx.x;
            const bool active = j < n_here;
            shade_slot(s, p, w, level, next, next_start, active, L.start + (active ? s_idx[j] : 0u));
        }
        __syncthreads();   // s_idx and the counts are reused by the next window
    }
}

template <int ACCEL, int MODE>
__global__ void __launch_bounds__(128) k_wave_shadow(DevScene s, WaveState w, int level) {
    const uint32_t n = min(w.levels[level].shadow_count, w.shadow_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const ShadowRec sr = w.shadows[i];
        Ray r;
        r.o = V3{sr.ox, sr.oy, sr.oz};
        r.d = V3{sr.dx, sr.dy, sr.dz};
        r.depth = 0;
        r.exclude = sr.exclude;
        if (scene_occ<ACCEL, MODE>(s, r, sr.dist)) atomicOr(&w.nodes[sr.node].occluded, 1u << (sr.j & 31u));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&w.counters[1], (unsigned long long)n);
}

// persistent FAST-BVH versions of extend and shadow (work items: the level's rays / shadow rays)
struct WaveLane {
    uint32_t idx;
};
struct ExtendWork {
    WaveState w;
    Level L;
    uint32_t *ctr;
    __device__ uint32_t total() const { return L.count; }
    __device__ uint32_t *counter() const { return ctr; }
    template <class L>
    __device__ const DevScene &scene(const L &, const DevScene &s) const { return s; }
    template <class L>
    __device__ const DevScene &view(const L &, const DevScene &s) const { return s; }
    __device__ bool begin(uint32_t item, WaveLane &lane, Ray &r) const {
        lane.idx = L.start + item;
        r = ray_of(w.rays[lane.idx]);
        return true;
    }
    __device__ bool finish(WaveLane &lane, Ray &, bool hit, float t, uint32_t id, const FastTrav &) const {
        w.nodes[lane.idx].hit_t = t;
        w.nodes[lane.idx].hit_id = hit ? id : MRT_HIT_NONE;
        return false;
    }
};
struct ShadowWork {
    WaveState w;
    uint32_t n;
    uint32_t *ctr;
    __device__ uint32_t total() const { return n; }
    __device__ uint32_t *counter() const { return ctr; }
    template <class L>
    __device__ const DevScene &scene(const L &, const DevScene &s) const { return s; }
    template <class L>
    __device__ const DevScene &view(const L &, const DevScene &s) const { return s; }
    __device__ bool begin(uint32_t item, WaveLane &lane, Ray &r, float &dist) const {
        const ShadowRec sr = w.shadows[item];
        lane.idx = item;
        r.o = V3{sr.ox, sr.oy, sr.oz};
        r.d = V3{sr.dx, sr.dy, sr.dz};
        r.depth = 0;
        r.exclude = sr.exclude;
        dist = sr.dist;
        return true;
    }
    __device__ void finish(WaveLane &lane, bool occluded) const {
        if (occluded) {
            const ShadowRec &sr = w.shadows[lane.idx];
            atomicOr(&w.nodes[sr.node].occluded, 1u << (sr.j & 31u));
        }
    }
};

// resident blocks of 128 threads per SM for the wavefront's persistent extend and shadow kernels
// (7 blocks, 72 registers: terrain PathTracer 1387 Mrays/s against 1325 at 8 and 1373 at 6)
#ifndef MRT_WAVE_BLOCKS_PER_SM
#define MRT_WAVE_BLOCKS_PER_SM 7
#endif
constexpr int kWaveBlocksPerSm = MRT_WAVE_BLOCKS_PER_SM;

template <int Q = kNodeQuorum>
__global__ void __launch_bounds__(128, kWaveBlocksPerSm) k_wave_extend_fast(DevScene s, WaveState w, int level, uint32_t *ctr) {
    const Level L = clamp_level(w, w.levels[level]);
    ExtendWork work{w, L, ctr};
    WaveLane lane;
    persistent_closest<false, Q>(s, work, lane);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&w.counters[0], (unsigned long long)L.count);
}

__global__ void __launch_bounds__(128, kGridBlocksPerSm) k_wave_extend_grid(DevScene s, WaveState w, int level, uint32_t *ctr) {
    const Level L = clamp_level(w, w.levels[level]);
    ExtendWork work{w, L, ctr};
    WaveLane lane;
    persistent_grid_closest(s, work, lane);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&w.counters[0], (unsigned long long)L.count);
}

__global__ void __launch_bounds__(128, kWaveBlocksPerSm) k_wave_shadow_fast(DevScene s, WaveState w, int level, uint32_t *ctr) {
    const uint32_t n = min(w.levels[level].shadow_count, w.shadow_cap);
    ShadowWork work{w, n, ctr};
    WaveLane lane;
    persistent_any(s, work, lane);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&w.counters[1], (unsigned long long)n);
}

// whole camera paths in one persistent launch (mrt_paths.cuh): work item = the wave's path i
struct WavePathWork {
    const DevScene *s;
    const RenderParams *p;
    WaveState w;
    uint32_t *ctr;
    __device__ uint32_t total() const { return w.n_roots; }
    __device__ uint32_t *counter() const { return ctr; }
    __device__ const DevScene &scene(const PathLane &) const { return *s; }
    __device__ const DevScene &view(const PathLane &) const { return *s; }
    __device__ const RenderParams &params(const PathLane &) const { return *p; }
    __device__ void begin(uint32_t item, PathLane &L, Ray &r) const {
        Task k;
        uint32_t pixel, sample;
        root_task(*p, w, item, k, pixel, sample);
        L.st = make_stream(p->seed, pixel, sample, p->strata, p->constant_value);
        r = primary_ray(*p, k, L.st);
        L.item = item;
        L.top = 1;
        L.fr[0].code = 1u;
        L.fr[0].depth = 1;
        L.fr[0].slot = 0;
    }
    __device__ void deliver(const PathLane &L, V3 rgb, bool flag) const {
        w.root_rgb[L.item] = make_float4(rgb.x, rgb.y, rgb.z, flag ? 1.0f : 0.0f);
    }
    __device__ void count(uint32_t n_closest, uint32_t n_shadow) const {
        const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, n_closest), d = __reduce_add_sync(0xFFFFFFFFu, n_shadow);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&w.counters[0], (unsigned long long)c);
            atomicAdd(&w.counters[1], (unsigned long long)d);
        }
    }
};

__global__ void __launch_bounds__(128, 8) k_wave_paths(DevScene s, RenderParams p, WaveState w, uint32_t *ctr) {
    WavePathWork work{&s, &p, w, ctr};
    persistent_paths(work);
}

// bottom-up evaluation of one level: the shade() bodies after their recursive calls return
__global__ void __launch_bounds__(128) k_wave_resolve(DevScene s, RenderParams p, WaveState w, int level) {
    const Level L = clamp_level(w, w.levels[level]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.count; i += gridDim.x * blockDim.x) {
        const uint32_t idx = L.start + i;
        const NodeRec &nd = w.nodes[idx];
        const RayRec &rr = w.rays[idx];
        V3 rgb{0.0f, 0.0f, 0.0f};
        bool flag = false;
        const uint32_t kind = nd.flags & 3u;
        if (kind == kEmit) {
            rgb = nd.point;
            flag = true;
        } else if (kind == kShaded) {   // misses and cut nodes are black
            Task k;
            uint32_t pixel, sample;
            root_task(p, w, rr.root, k, pixel, sample);
            const Stream st = make_stream(p.seed, pixel, sample, p.strata, p.constant_value);
            resolve_node(s, p, nd, rr, st, rgb, flag);
        }
        if (rr.parent == 0xFFFFFFFFu) {
            w.root_rgb[rr.root] = make_float4(rgb.x, rgb.y, rgb.z, flag ? 1.0f : 0.0f);
        } else {
            NodeRec &pn = w.nodes[rr.parent];
            pn.child[rr.slot] = rgb;
            if (flag) atomicOr(&pn.child_flag, 1u << rr.slot);
        }
    }
}

// fold the wave's per-sample values into the bitmap in sample order (Renderer.cpp:105-107)
__global__ void k_wave_accumulate(RenderParams p, WaveState w) {
    const uint32_t g0 = w.root_first, g1 = w.root_first + w.n_roots;
    const uint32_t t0 = g0 / p.spp, t1 = (g1 - 1) / p.spp;
    for (uint32_t t = t0 + blockIdx.x * blockDim.x + threadIdx.x; t <= t1; t += gridDim.x * blockDim.x) {
        const Task k = task_of(p, p.task_base + t);
        const int64_t slot = p.accum ? accum_slot(p, k) : -1;
        uint32_t bm = p.bitmap[k.index];
        float4 acc = slot >= 0 ? p.accum[slot] : make_float4(0, 0, 0, 0);
        const uint32_t a = max(g0, t * p.spp), b = min(g1, (t + 1) * p.spp);
        for (uint32_t g = a; g < b; ++g) {
            const float4 c = w.root_rgb[g - g0];
            const V3 rgb{c.x, c.y, c.z};
            const uint32_t sample = p.spp_offset + (g - t * p.spp);
            bm = incremental_avg(rgb, bm, sample + 1u);
            acc.x += rgb.x; acc.y += rgb.y; acc.z += rgb.z; acc.w += 1.0f;
        }
        p.bitmap[k.index] = bm;
        if (slot >= 0) p.accum[slot] = acc;
    }
}

// ============================== host orchestration ============================================
struct TaskPlan {
    uint32_t width = 0, height = 0, stride_px = 0;
    bool uploaded = false;               // explicit list already in the scene's work[0]
    bool implicit = true;
    uint32_t n_tasks = 0;
    std::vector<Task> list;                  // explicit tasks, block order
    std::vector<uint32_t> round_first, round_count;
};

// Renderer ctor (Renderer.cpp:12-29) + renderScene block arithmetic (Renderer.cpp:79-93)
bool plan_tasks(const MrtRenderOpts &o, uint32_t stride_px, TaskPlan &plan) {
    const uint32_t w = o.width, h = o.height;
    const uint32_t bsx = w / 16u, bsy = h / 16u;
    if (bsx == 0 || bsy == 0) return false;
    const uint32_t domain = (w / bsx) * (h / bsy);
    const uint64_t res = (uint64_t)w * h;
    std::vector<Task> tasks;
    tasks.reserve((size_t)256 * bsx * bsy);
    for (uint32_t i = 0; i < 256; ++i) {
        const float block = halton(i, 2);
        const uint32_t rb = (uint32_t)roundf(block * (float)domain);
        const uint32_t pixel = (uint32_t)(((uint64_t)rb * bsx) % res);
        const uint32_t sy = ((pixel / w) * bsy) % h;
        for (uint32_t y = sy; y < sy + bsy; ++y) {
            const uint32_t yw = y * stride_px;
            const uint32_t sx = (pixel + yw) % w;
            for (uint32_t x = sx; x < sx + bsx; ++x) tasks.push_back(Task{x, y, yw + x});
        }
    }
    // the implicit rectangle?
    const uint32_t rows = 16u * bsy;
    bool rect = tasks.size() == (size_t)w * rows;
    std::vector<uint8_t> seen((size_t)stride_px * h + 1, 0);
    if (rect) {
        for (const Task &t : tasks) {
            if (t.x >= w || t.y >= rows || t.index != t.y * stride_px + t.x || seen[t.index]) { rect = false; break; }
            seen[t.index] = 1;
        }
    }
    if (rect) {
        plan.implicit = true;
        plan.n_tasks = w * rows;
        plan.round_first = {0};
        plan.round_count = {plan.n_tasks};
        return true;
    }
    // explicit: drop tasks outside the bitmap (undefined behaviour in the reference), then rounds
    // in which every pixel appears at most once, preserving block order per pixel
    plan.implicit = false;
    std::vector<uint32_t> visits((size_t)stride_px * h + 1, 0);
    std::vector<std::vector<Task>> rounds;
    for (const Task &t : tasks) {
        if ((uint64_t)t.index >= (uint64_t)stride_px * h) continue;   // outside the bitmap
        const uint32_t r = visits[t.index]++;
        if (rounds.size() <= r) rounds.emplace_back();
        rounds[r].push_back(t);
    }
    for (auto &r : rounds) {
        plan.round_first.push_back((uint32_t)plan.list.size());
        plan.round_count.push_back((uint32_t)r.size());
        plan.list.insert(plan.list.end(), r.begin(), r.end());
    }
    plan.n_tasks = (uint32_t)plan.list.size();
    return true;
}

TaskPlan *cached_plan(MrtScene *s, uint32_t w, uint32_t h, uint32_t stride_px) {
    TaskPlan *p = static_cast<TaskPlan *>(s->plan_cache);
    if (p && p->width == w && p->height == h && p->stride_px == stride_px) return p;
    delete p;
    p = new TaskPlan();
    p->width = w;
    p->height = h;
    p->stride_px = stride_px;
    MrtRenderOpts o{};
    o.width = w;
    o.height = h;
    if (!plan_tasks(o, stride_px, *p)) p->n_tasks = 0;
    s->plan_cache = p;
    s->plan_cache_free = [](void *q) { delete static_cast<TaskPlan *>(q); };
    return p;
}

template <int ACCEL, int MODE>
void launch_noshadows(const DevScene &s, const RenderParams &p, uint32_t first, uint32_t count, int grid, cudaStream_t q) {
    k_render_noshadows<ACCEL, MODE><<<grid, 128, 0, q>>>(s, p, first, count);
}

template <int ACCEL, int MODE>
void launch_wave_level(const DevScene &s, const RenderParams &p, const WaveState &w, int level, int grid, cudaStream_t q,
                       uint32_t *ctrs) {
    if (ACCEL == MRT_ACCEL_BVH && MODE == MRT_BVH_FAST) {
        // counters [2 * level] and [2 * level + 1] were zeroed for this wave
        // one quorum for every level: 16 for the camera rays of level 0 made the terrain PathTracer
        // 0.4 % slower and the 256-job batch 0.4 % faster
        k_wave_extend_fast<kNodeQuorum><<<grid, 128, 0, q>>>(s, w, level, ctrs + 2 * level);
        if (w.sort_shading) k_wave_shade_sorted<<<grid, 128, 0, q>>>(s, p, w, level);
        else k_wave_shade<<<grid, 128, 0, q>>>(s, p, w, level);
        k_wave_shadow_fast<<<grid, 128, 0, q>>>(s, w, level, ctrs + 2 * level + 1);
        return;
    }
    if (ACCEL == MRT_ACCEL_REGULAR_GRID) k_wave_extend_grid<<<grid, 128, 0, q>>>(s, w, level, ctrs + 2 * level);
    else k_wave_extend<ACCEL, MODE><<<grid, 128, 0, q>>>(s, w, level);
    if (w.sort_shading) k_wave_shade_sorted<<<grid, 128, 0, q>>>(s, p, w, level);
    else k_wave_shade<<<grid, 128, 0, q>>>(s, p, w, level);
    k_wave_shadow<ACCEL, MODE><<<grid, 128, 0, q>>>(s, w, level);
}

#define MRT_DISPATCH(fn, accel, mode, ...)                                                                 \
    do {                                                                                                    \
        if ((accel) == MRT_ACCEL_NAIVE) fn<MRT_ACCEL_NAIVE, MRT_BVH_FAST>(__VA_ARGS__);                     \
        else if ((accel) == MRT_ACCEL_REGULAR_GRID) fn<MRT_ACCEL_REGULAR_GRID, MRT_BVH_FAST>(__VA_ARGS__);  \
        else if ((mode) == MRT_BVH_REFERENCE) fn<MRT_ACCEL_BVH, MRT_BVH_REFERENCE>(__VA_ARGS__);            \
        else fn<MRT_ACCEL_BVH, MRT_BVH_FAST>(__VA_ARGS__);                                                  \
    } while (0)

// Renderer::stopRender seen between waves: the work already queued finishes (the caller's buffers
// stay in use until then), the bitmap keeps the samples folded so far
int cancelled(MrtContext *ctx, cudaStream_t q) {
    cudaStreamSynchronize(q);
    set_error(ctx, "render stopped (mrt_render_stop)");
    return MRT_ERR_CANCELLED;
}

// Renders of at most this many camera paths per pass run as whole-path launches, larger ones as the
// level-by-level wavefront (MRT_PATHS_MAX; 0 = always the wavefront).  Measured on one B200: a
// 256x256 Whitted frame 3.1x faster whole-path (launch-bound), a 512x512x4 PathTracer soup 1.2x
// faster, a 1024x1024 terrain 1.1-1.3x slower (the wavefront's per-level coherence wins there).
uint64_t paths_max_setting() {
    static uint64_t v = [] {
        const char *e = getenv("MRT_PATHS_MAX");
        return e ? (uint64_t)atoll(e) : (uint64_t)(1u << 19);
    }();
    return v;
}

uint32_t wave_roots_setting() {
    static uint32_t v = [] {
        const char *e = getenv("MRT_WAVE_ROOTS");
        const long x = e ? atol(e) : (1l << 21);
        return (uint32_t)std::max(1024l, std::min(x, 1l << 25));
    }();
    return v;
}

}  // namespace

namespace mrt_host {

static int render_impl(MrtScene *s, const MrtCamera *cam, const MrtRenderOpts *o, uint32_t *d_bitmap, uint32_t stride,
                       float *d_accum, MrtRenderStats *stats, uint32_t strata, HostOut *out) {
    MrtContext *ctx = s->ctx;
    cudaStream_t q = ctx->stream;
    const uint32_t stride_px = stride / 4u;
    // the block schedule depends only on (width, height, row pitch): planned once per scene
    TaskPlan &plan = *cached_plan(s, o->width, o->height, stride_px);
    if (plan.n_tasks == 0) {
        set_error(ctx, "mrt_render: width and height must be at least 16 (Renderer block size width/16)");
        return MRT_ERR_ARG;
    }
    RenderParams p{};
    p.cam = make_camera(*cam);
    p.width = o->width; p.height = o->height; p.spp = o->spp; p.spl = o->spl; p.stride_px = stride_px;
    p.pixel_sampler = o->pixel_sampler; p.light_sampler = o->light_sampler; p.rr_sampler = o->rr_sampler;
    p.shader = o->shader; p.constant_value = o->constant_value;
    p.depth_min = o->depth_min; p.depth_max = o->depth_max;
    p.seed = o->seed; p.spp_offset = o->spp_offset;
    p.strata = strata;
    p.bitmap = d_bitmap;
    p.accum = (float4 *)d_accum;
    p.inv_w = 1.0f / (float)o->width;   // Renderer.cpp:68-71
    p.inv_h = 1.0f / (float)o->height;
    p.pw = 0.5f / (float)o->width;
    p.ph = 0.5f / (float)o->height;
    p.depth_point = V3{o->depth_point[0], o->depth_point[1], o->depth_point[2]};
    p.n_tasks = plan.n_tasks;
    int st = MRT_OK;
    if (!plan.implicit) {
        if (!plan.uploaded) {
            st = ensure(ctx, s->work[0], sizeof(Task) * plan.list.size());
            if (st == MRT_OK)
                st = cuda_status(ctx, cudaMemcpyAsync(s->work[0].ptr, plan.list.data(), sizeof(Task) * plan.list.size(),
                                                      cudaMemcpyHostToDevice, q), "tasks");
            if (st != MRT_OK) return st;
            plan.uploaded = true;
        }
        p.tasks = (const Task *)s->work[0].ptr;
    }
    if (plan.round_first.size() > 1 && o->spp > 1) {
        // pixels revisited within a pass: the reference's pass-major order, one pass at a time
        MrtRenderStats total{0, 0, 0, 0.0f, 0.0f, 0u, 0u};
        for (uint32_t si = 0; si < o->spp; ++si) {
            MrtRenderOpts one = *o;
            one.spp = 1;
            one.spp_offset = o->spp_offset + si;
            MrtRenderStats part{};
            st = render_impl(s, cam, &one, d_bitmap, stride, d_accum, &part, strata, nullptr);
            if (st != MRT_OK) return st;
            total.rays_closest += part.rays_closest;
            total.rays_shadow += part.rays_shadow;
            total.paths += part.paths;
            total.device_ms += part.device_ms;
            total.trace_ms += part.trace_ms;
            total.kernel_launches += part.kernel_launches;
        }
        if (stats) *stats = total;
        return MRT_OK;
    }
    const int accel = s->opts.accelerator, mode = s->opts.bvh_mode;
    const int grid = ctx->sm_count * 16;
    uint64_t rays_closest = 0, rays_shadow = 0;
    uint32_t launches = 0;   // kernels launched by this render
    float trace_ms = 0.0f;
    int trace_pairs = 0;   // recorded pairs of ctx->trace_ev not yet added to trace_ms
    auto add_trace_time = [&]() {
        if (trace_pairs > 0 && cudaEventSynchronize(ctx->trace_ev[2 * trace_pairs - 1]) == cudaSuccess)
            for (int k = 0; k < trace_pairs; ++k) {
                float t = 0.0f;
                if (cudaEventElapsedTime(&t, ctx->trace_ev[2 * k], ctx->trace_ev[2 * k + 1]) == cudaSuccess) trace_ms += t;
            }
        trace_pairs = 0;
    };
    s->progress.store(0);
    cudaEventRecord(ctx->ev0, q);
    if (direct_shader(o->shader)) {
        const bool fast = accel == MRT_ACCEL_BVH && mode == MRT_BVH_FAST;
        const uint32_t rows = 16u * (o->height / 16u);
        const uint32_t tiles_x = (plan.implicit && o->width % 2u == 0 && rows % 16u == 0) ? o->width / 2u : 0u;
        for (size_t r = 0; r < plan.round_first.size(); ++r) {
            if (s->stop.load()) return cancelled(ctx, q);
            if ((fast || accel == MRT_ACCEL_REGULAR_GRID) && kNsSplit) {
                // chunks of at most kNsChunk (sample, pixel) items: whole samples of up to kNsChunk pixels.
                // A frame into page-locked host buffers that is one chunk (the plain rectangle, whole
                // 16-row stripes) is traced in one launch and shaded in up to kHostBands bands of whole
                // stripes, so that the copies out overlap the shading.  (Tracing it in bands as well was
                // slower end to end on the 1080p soup frame, 1121 against 1496 Mrays/s: each shorter
                // traversal launch pays its own tail.)
                const uint32_t count = plan.round_count[r];
                const uint32_t n_pix_max = std::min<uint32_t>(count, kNsChunk);
                const uint32_t stripe = 16u * o->width;
                uint32_t band_rows = 0;   // items per band (0: one shading launch per pass, no copies here)
                if (kHostBandsOn && out && out->bitmap && plan.implicit && plan.round_first.size() == 1 && plan.round_first[0] == 0 &&
                    stride == 4u * o->width && count <= kNsChunk && count % stripe == 0 && count / stripe >= 2) {
                    const uint32_t stripes = count / stripe;
                    const uint32_t bands = std::min<uint32_t>(stripes, MrtContext::kHostBands);
                    band_rows = ((stripes + bands - 1) / bands) * stripe;
                }
                st = ensure(ctx, ctx->wave[1], sizeof(uint2) * (size_t)kNsChunk);
                if (st != MRT_OK) return st;
                uint2 *hits = (uint2 *)ctx->wave[1].ptr;
                for (uint32_t j0 = 0; j0 < count; j0 += n_pix_max) {
                    const uint32_t n_pix = std::min(n_pix_max, count - j0);
                    const uint32_t per = std::max(1u, kNsChunk / n_pix);
                    for (uint32_t s0 = 0; s0 < o->spp; s0 += per) {
                        if (s->stop.load()) return cancelled(ctx, q);
                        const uint32_t n_s = std::min(per, o->spp - s0);
                        NsTraceWork tw{nullptr, plan.round_first[r], j0, n_pix, s0, n_pix * n_s, tiles_x, ctx->d_counters, hits};
                        cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t), q);
                        if (trace_pairs == MrtContext::kTraceEvents) add_trace_time();
                        cudaEventRecord(ctx->trace_ev[2 * trace_pairs], q);
                        if (fast) k_ns_trace<<<ctx->sm_count * kNsBlocksPerSm, 128, 0, q>>>(s->dev, tw, p);
                        else k_ns_trace_grid<<<ctx->sm_count * kGridBlocksPerSm, 128, 0, q>>>(s->dev, tw, p);
                        cudaEventRecord(ctx->trace_ev[2 * trace_pairs + 1], q);
                        ++trace_pairs;
                        launches += 2;
                        if (!band_rows || s0 + n_s < o->spp) {
                            k_ns_shade<<<(n_pix + 127) / 128, 128, 0, q>>>(s->dev, p, plan.round_first[r], j0, n_pix, s0,
                                                                            n_s, tiles_x, hits, n_pix);
                            continue;
                        }
                        // the last samples of the frame: shaded band by band, each band's rows going to
                        // the host on the copy stream while the next band is shaded
                        launches -= 1;
                        for (uint32_t b0 = 0; b0 < n_pix && st == MRT_OK; b0 += band_rows) {
                            const uint32_t nb = std::min(band_rows, n_pix - b0);
                            const int slot = (int)(b0 / band_rows);
                            k_ns_shade<<<(nb + 127) / 128, 128, 0, q>>>(s->dev, p, plan.round_first[r], j0 + b0, nb, s0,
                                                                         n_s, tiles_x, hits + b0, n_pix);
                            ++launches;
                            st = cuda_status(ctx, cudaEventRecord(ctx->band_ev[slot], q), "band event");
                            if (st == MRT_OK)
                                st = cuda_status(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->band_ev[slot], 0), "band wait");
                            if (st == MRT_OK) {
                                out->queued = true;
                                st = cuda_status(ctx, cudaMemcpyAsync(out->bitmap + b0, d_bitmap + b0, 4ull * nb,
                                                                      cudaMemcpyDeviceToHost, ctx->copy_stream), "band out");
                            }
                            if (st == MRT_OK && out->accum && d_accum)
                                st = cuda_status(ctx, cudaMemcpyAsync(out->accum + 4ull * b0, d_accum + 4ull * b0, 16ull * nb,
                                                                      cudaMemcpyDeviceToHost, ctx->copy_stream), "band sums out");
                        }
                        if (st != MRT_OK) return st;
                        out->rows_done = true;
                    }
                }
            } else if (fast) {
                cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t), q);
                k_render_noshadows_fast<<<ctx->sm_count * kNsBlocksPerSm, 128, 0, q>>>(s->dev, p, plan.round_first[r],
                                                                         plan.round_count[r], ctx->d_counters, tiles_x);
                ++launches;
            } else if (accel == MRT_ACCEL_REGULAR_GRID) {
                cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t), q);
                k_render_noshadows_grid<<<ctx->sm_count * kGridBlocksPerSm, 128, 0, q>>>(s->dev, p, plan.round_first[r],
                                                                         plan.round_count[r], ctx->d_counters, tiles_x);
                ++launches;
            } else {
                MRT_DISPATCH(launch_noshadows, accel, mode, s->dev, p, plan.round_first[r], plan.round_count[r], grid, q);
                ++launches;
            }
        }
        rays_closest = (uint64_t)plan.n_tasks * o->spp;
    } else {
        if (o->spl > 32) { set_error(ctx, "mrt_render: samplesLight above 32 is not supported by the wavefront"); return MRT_ERR_ARG; }
        uint64_t all_roots = 0;
        for (uint32_t c : plan.round_count) all_roots += (uint64_t)c * o->spp;
        const bool paths = all_roots <= paths_max_setting() && accel == MRT_ACCEL_BVH && mode == MRT_BVH_FAST &&
                           o->depth_max >= 0 && o->depth_max + 1 <= kPathFrames;
        uint64_t max_round = 0;
        for (uint32_t c : plan.round_count) max_round = std::max<uint64_t>(max_round, c);
        const uint32_t wave = (uint32_t)std::min<uint64_t>(max_round * o->spp,
                                                           paths ? std::max(wave_roots_setting(), 1u << 22)
                                                                 : wave_roots_setting());
        const int levels = std::max(1, o->depth_max + 1);
        const uint64_t ray_cap = paths ? 0 : (uint64_t)wave * (uint64_t)(levels + 2);
        const uint64_t shadow_cap = paths ? 0 : (uint64_t)wave * std::max(1u, o->spl) * 2ull;
        if (ray_cap > 0xFFFFFFF0ull) { set_error(ctx, "mrt_render: wave too large"); return MRT_ERR_ARG; }
        if (2 * (levels + 1) > 64) { set_error(ctx, "mrt_render: depth_max above 30"); return MRT_ERR_ARG; }
        if (!paths) {   // the wavefront's queues (whole-path launches keep their state per lane)
            if (st == MRT_OK) st = ensure(ctx, ctx->wave[1], sizeof(RayRec) * ray_cap);
            if (st == MRT_OK) st = ensure(ctx, ctx->wave[2], sizeof(NodeRec) * ray_cap);
            if (st == MRT_OK) st = ensure(ctx, ctx->wave[3], sizeof(ShadowRec) * shadow_cap);
        }
        if (st == MRT_OK) st = ensure(ctx, ctx->wave[4], sizeof(Level) * (levels + 2));
        if (st == MRT_OK) st = ensure(ctx, ctx->wave[5], sizeof(float4) * wave);
        if (st == MRT_OK) st = ensure(ctx, ctx->wave[6], 16);
        if (st != MRT_OK) return st;
        WaveState w{};
        w.rays = (RayRec *)ctx->wave[1].ptr;
        w.nodes = (NodeRec *)ctx->wave[2].ptr;
        w.shadows = (ShadowRec *)ctx->wave[3].ptr;
        w.levels = (Level *)ctx->wave[4].ptr;
        w.root_rgb = (float4 *)ctx->wave[5].ptr;
        w.counters = (unsigned long long *)ctx->wave[6].ptr;
        w.ray_cap = (uint32_t)ray_cap;
        w.shadow_cap = (uint32_t)shadow_cap;
        // per-material shade queues where the scene mixes diffuse with mirror / glass materials
        w.sort_shading = (o->flags & MRT_RENDER_SHADE_QUEUES) && s->mixed_materials ? 1u : 0u;
        cudaMemsetAsync(w.counters, 0, 16, q);
        // at most one wave queued ahead of the one running: a stop request ends the render within two
        // waves, and progress counts finished waves
        uint64_t waves_issued = 0;
        uint64_t done_samples[2] = {0, 0};
        for (size_t rd = 0; rd < plan.round_first.size(); ++rd) {
            p.task_base = plan.round_first[rd];
            const uint64_t total_roots = (uint64_t)plan.round_count[rd] * o->spp;
            for (uint64_t r0 = 0; r0 < total_roots; r0 += wave) {
                if (waves_issued >= 2) {
                    const int slot = (int)(waves_issued % 2);
                    st = cuda_status(ctx, cudaEventSynchronize(ctx->wave_ev[slot]), "render");
                    if (st != MRT_OK) return st;
                    s->progress.store((uint32_t)done_samples[slot]);
                }
                if (s->stop.load()) return cancelled(ctx, q);
                w.root_first = (uint32_t)r0;
                w.n_roots = (uint32_t)std::min<uint64_t>(wave, total_roots - r0);
                if (paths) {
                    cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t), q);
                    k_wave_paths<<<ctx->sm_count * 8, 128, 0, q>>>(s->dev, p, w, ctx->d_counters);
                    launches += 2;   // with the fold below
                } else {
                    cudaMemsetAsync(w.levels, 0, sizeof(Level) * (levels + 2), q);
                    cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t) * 2 * (levels + 1), q);
                    k_wave_raygen<<<grid, 128, 0, q>>>(p, w);
                    for (int b = 0; b < levels; ++b)
                        MRT_DISPATCH(launch_wave_level, accel, mode, s->dev, p, w, b, grid, q, ctx->d_counters);
                    for (int b = levels - 1; b >= 0; --b) k_wave_resolve<<<grid, 128, 0, q>>>(s->dev, p, w, b);
                    launches += 2u + 4u * (uint32_t)levels;   // raygen, per level extend / shade / shadow /
                                                              // resolve, the fold below
                }
                k_wave_accumulate<<<grid, 128, 0, q>>>(p, w);
                const int slot = (int)(waves_issued % 2);
                cudaEventRecord(ctx->wave_ev[slot], q);
                done_samples[slot] = (r0 + w.n_roots) / std::max<uint64_t>(1, plan.round_count[rd]);
                ++waves_issued;
            }
        }
        unsigned long long cnt[2] = {0, 0};
        st = cuda_status(ctx, cudaMemcpyAsync(cnt, w.counters, 16, cudaMemcpyDeviceToHost, q), "counters");
        if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "render");
        rays_closest = cnt[0];
        rays_shadow = cnt[1];
    }
    cudaEventRecord(ctx->ev1, q);
    if (st == MRT_OK) st = cuda_status(ctx, cudaGetLastError(), "render kernels");
    if (st == MRT_OK) st = cuda_status(ctx, cudaEventSynchronize(ctx->ev1), "render");
    if (st == MRT_OK) st = check_kernel_error(ctx);
    s->progress.store(o->spp);
    add_trace_time();
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->rays_closest = rays_closest;
        stats->rays_shadow = rays_shadow;
        stats->paths = (uint64_t)plan.n_tasks * o->spp;
        stats->device_ms = ms;
        stats->trace_ms = trace_ms;
        stats->kernel_launches = launches;
        stats->reserved = 0;
    }
    return st;
}

int render(MrtScene *s, const MrtCamera *cam, const MrtRenderOpts *o, uint32_t *d_bitmap, uint32_t stride,
           float *d_accum, MrtRenderStats *stats, HostOut *out) {
    return render_impl(s, cam, o, d_bitmap, stride, d_accum, stats, o->spp, out);
}

}  // namespace mrt_host

// host memory that the driver has page-locked (cudaHostAlloc / cudaHostRegister): device copies into it
// are asynchronous
static bool page_locked(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

extern "C" {

int mrt_render(MrtScene *s, const MrtCamera *cam, const MrtRenderOpts *o, uint32_t *bitmap, uint32_t stride_bytes,
               float *accum, uint32_t mem, MrtRenderStats *stats) {
    if (!s || !cam || !o || !bitmap) return MRT_ERR_ARG;
    MrtContext *ctx = s->ctx;
    if (!s->built) { set_error(ctx, "mrt_render before mrt_scene_build"); return MRT_ERR_STATE; }
    if (o->shader < MRT_SHADER_NOSHADOWS || o->shader > MRT_SHADER_DIFFUSE || o->spp == 0 ||
        (o->spl == 0 && (o->shader == MRT_SHADER_WHITTED || o->shader == MRT_SHADER_PATHTRACER || o->shader == MRT_SHADER_NOSHADOWS)) ||
        o->width < 16 || o->height < 16 || stride_bytes < 4u * o->width || (cam->kind != MRT_CAMERA_PERSPECTIVE && cam->kind != MRT_CAMERA_ORTHOGRAPHIC) ||
        o->pixel_sampler < 0 || o->pixel_sampler > 3 || o->light_sampler < 0 || o->light_sampler > 3 ||
        o->rr_sampler < 0 || o->rr_sampler > 3) {
        set_error(ctx, "mrt_render: invalid options");
        return MRT_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    s->stop.store(0);
    const size_t bm_bytes = (size_t)stride_bytes * o->height;
    const size_t acc_bytes = 16ull * o->width * o->height;
    const size_t acc_offset = (bm_bytes + 255) & ~(size_t)255;   // the sums are read as float4
    uint32_t *d_bitmap = bitmap;
    float *d_accum = accum;
    int st = MRT_OK;
    if (mem == MRT_MEM_DEVICE && (((uintptr_t)bitmap & 3u) || ((uintptr_t)accum & 15u) || (stride_bytes & 3u))) {
        set_error(ctx, "mrt_render: the bitmap must be 4-byte aligned (and the row pitch a multiple of 4) and the "
                       "sums 16-byte aligned");
        return MRT_ERR_ARG;
    }
    HostOut out;
    size_t rows_bytes = bm_bytes, acc_rows = accum ? acc_bytes : 0;   // what the render can change
    if (mem == MRT_MEM_HOST) {
        st = ensure(ctx, ctx->wave[7], acc_offset + (accum ? acc_bytes : 0));
        if (st != MRT_OK) return st;
        d_bitmap = (uint32_t *)ctx->wave[7].ptr;
        d_accum = accum ? (float *)((char *)ctx->wave[7].ptr + acc_offset) : nullptr;
        // On the plain rectangle (row pitch = 4 * width) the block schedule is the first n_tasks pixels,
        // whole rows (the height mod 16 rows below it are never rendered, Renderer.cpp:20-21): only those
        // go in and out, and the caller's other rows stay as they are.  The first samples of a frame
        // (spp_offset 0) replace every pixel they render without reading it (incrementalAvg with n = 1
        // keeps nothing of the old value, Utils.cpp:48-70): then no bitmap byte goes in.
        bool plain = false;
        if (stride_bytes == 4u * o->width) {
            const TaskPlan &plan = *cached_plan(s, o->width, o->height, o->width);
            plain = plan.n_tasks > 0 && plan.implicit;
            if (plain) {
                rows_bytes = 4ull * plan.n_tasks;
                if (accum) acc_rows = 16ull * plan.n_tasks;
            }
        }
        const size_t in_bytes = (plain && o->spp_offset == 0) ? 0 : rows_bytes;
        if (in_bytes)
            st = cuda_status(ctx, cudaMemcpyAsync(d_bitmap, bitmap, in_bytes, cudaMemcpyHostToDevice, ctx->stream), "bitmap in");
        if (st == MRT_OK && accum)
            st = cuda_status(ctx, cudaMemcpyAsync(d_accum, accum, acc_rows, cudaMemcpyHostToDevice, ctx->stream), "accum in");
        if (st != MRT_OK) return st;
        // page-locked buffers: the render may copy finished bands out while it shades the rest (a copy
        // into pageable memory would return only when done, holding up the launches behind it)
        if (plain && page_locked(bitmap) && (!accum || page_locked(accum))) {
            out.bitmap = bitmap;
            out.accum = accum;
        }
    }
    st = render(s, cam, o, d_bitmap, stride_bytes, d_accum, stats, out.bitmap ? &out : nullptr);
    if (mem == MRT_MEM_HOST) {
        if (st == MRT_OK && !out.rows_done) {
            st = cuda_status(ctx, cudaMemcpyAsync(bitmap, d_bitmap, rows_bytes, cudaMemcpyDeviceToHost, ctx->stream), "bitmap out");
            if (st == MRT_OK && accum)
                st = cuda_status(ctx, cudaMemcpyAsync(accum, d_accum, acc_rows, cudaMemcpyDeviceToHost, ctx->stream), "accum out");
            if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "render copy out");
        }
        if (out.queued) {   // copies of bands on the copy stream: done before the call returns, also on an error
            const int cs = cuda_status(ctx, cudaStreamSynchronize(ctx->copy_stream), "render band copies");
            if (st == MRT_OK) st = cs;
        }
    }
    return st;
}

void mrt_render_stop(MrtScene *s) {
    if (s) s->stop.store(1);
}

uint32_t mrt_render_progress(const MrtScene *s) { return s ? s->progress.load() : 0u; }

}  // extern "C"

// =============================================================================================
// mrt_render_noalloc: the same render with every piece of scratch in a fixed device array.
//
// For callers that cannot allocate device memory while they render: a process whose device memory
// is owned by another allocator or a fixed budget (an engine that lends the renderer a pool and
// forbids cudaMalloc), or a latency-critical thread that must not hit cudaMalloc / cudaFree's implicit
// synchronisation.  The caller passes device buffers for the bitmap and the sums; everything else the
// kernels need (work counters, the wave's ray / node / shadow queues, per-sample values) lives in
// g_noalloc_scratch below, which every GPU that loads the library holds until the process exits.
//
// Limits of this variant: image sizes whose block schedule is the plain rectangle (width a multiple
// of 16, row pitch = width, as the reference CLI sizes images), samplesLight <= kNoAllocMaxSpl,
// depth_max <= kNoAllocMaxDepth; waves of kNoAllocWave camera paths.  Larger requests fail with
// MRT_ERR_ARG.  The call returns once its work on the context's stream has finished (it waits on
// events and on the stream, as mrt_render does).  The first call on a device looks up the array's
// device address (cudaGetSymbolAddress); make that first call before any stream capture.  All calls
// share the array: calls that overlap on the GPU (two host threads, or two contexts on one device)
// race.  As in mrt_render, at most one wave is queued ahead of the running one, so mrt_render_stop
// ends the render within two waves and mrt_render_progress counts finished waves.
// =============================================================================================
namespace {

constexpr uint32_t kNoAllocWave = 4096;
constexpr int kNoAllocMaxDepth = 10;
constexpr uint32_t kNoAllocMaxSpl = 4;
constexpr int kNoAllocLevels = kNoAllocMaxDepth + 1;
constexpr size_t kNaCounters = 0;                                   // 64 x uint32 work counters
constexpr size_t kNaWaveCounters = 256;                             // 2 x uint64 ray counters
constexpr size_t kNaLevels = 512;                                   // Level x (levels + 2)
constexpr size_t kNaRoot = 1024;                                    // float4 x wave
constexpr size_t kNaRays = kNaRoot + 16ull * kNoAllocWave;
constexpr size_t kNaRayCap = (size_t)kNoAllocWave * (kNoAllocLevels + 2);
constexpr size_t kNaNodes = kNaRays + sizeof(RayRec) * kNaRayCap;
constexpr size_t kNaShadows = kNaNodes + sizeof(NodeRec) * kNaRayCap;
constexpr size_t kNaShadowCap = (size_t)kNoAllocWave * kNoAllocMaxSpl * 2;
constexpr size_t kNoAllocScratchBytes = (kNaShadows + sizeof(ShadowRec) * kNaShadowCap + 255) & ~(size_t)255;
static_assert(sizeof(Level) * (kNoAllocLevels + 2) <= kNaRoot - kNaLevels, "level table overlaps");
static_assert(kNoAllocScratchBytes <= 12u * 1024u * 1024u, "scratch above 12 MiB");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// device address of g_noalloc_scratch per device (looked up once, with that device current)
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {nullptr};

int noalloc_scratch(MrtContext *ctx, unsigned char **out) {
    if (ctx->device < 0 || ctx->device >= 64) { set_error(ctx, "mrt_render_noalloc: device index above 63"); return MRT_ERR_ARG; }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[ctx->device]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) return cuda_status(ctx, e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress");
        g_noalloc_ptr[ctx->device] = ptr;
    }
    *out = static_cast<unsigned char *>(g_noalloc_ptr[ctx->device]);
    return MRT_OK;
}

}  // namespace

extern "C" int mrt_render_noalloc(MrtScene *s, const MrtCamera *cam, const MrtRenderOpts *o, uint32_t *bitmap,
                                  uint32_t stride_bytes, float *accum, MrtRenderStats *stats) {
    if (!s || !cam || !o || !bitmap) return MRT_ERR_ARG;
    MrtContext *ctx = s->ctx;
    if (!s->built) { set_error(ctx, "mrt_render_noalloc before mrt_scene_build"); return MRT_ERR_STATE; }
    if (o->shader < MRT_SHADER_NOSHADOWS || o->shader > MRT_SHADER_DIFFUSE || o->spp == 0 ||
        (o->spl == 0 && (o->shader == MRT_SHADER_WHITTED || o->shader == MRT_SHADER_PATHTRACER || o->shader == MRT_SHADER_NOSHADOWS)) ||
        o->width < 16 || o->height < 16 || (cam->kind != MRT_CAMERA_PERSPECTIVE && cam->kind != MRT_CAMERA_ORTHOGRAPHIC) || o->pixel_sampler < 0 ||
        o->pixel_sampler > 3 || o->light_sampler < 0 || o->light_sampler > 3 || o->rr_sampler < 0 || o->rr_sampler > 3) {
        set_error(ctx, "mrt_render_noalloc: invalid options");
        return MRT_ERR_ARG;
    }
    const uint32_t bsy = o->height / 16u;
    if (o->width % 16u != 0 || stride_bytes != 4u * o->width || o->height / bsy != 16u) {
        set_error(ctx, "mrt_render_noalloc: width must be a multiple of 16 with row pitch = width and height / (height / 16) == 16");
        return MRT_ERR_ARG;
    }
    if (o->spl > kNoAllocMaxSpl || o->depth_max > kNoAllocMaxDepth || o->depth_max < 0) {
        set_error(ctx, "mrt_render_noalloc: samplesLight <= %u and 0 <= depth_max <= %d in this variant", kNoAllocMaxSpl,
                  kNoAllocMaxDepth);
        return MRT_ERR_ARG;
    }
    if (((uintptr_t)bitmap & 3u) || ((uintptr_t)accum & 15u)) {
        set_error(ctx, "mrt_render_noalloc: bitmap must be 4-byte aligned and the sums 16-byte aligned");
        return MRT_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    unsigned char *scratch = nullptr;
    int st = noalloc_scratch(ctx, &scratch);
    if (st != MRT_OK) return st;
    cudaStream_t q = ctx->stream;
    s->stop.store(0);
    RenderParams p{};
    p.cam = make_camera(*cam);
    p.width = o->width; p.height = o->height; p.spp = o->spp; p.spl = o->spl; p.stride_px = o->width;
    p.pixel_sampler = o->pixel_sampler; p.light_sampler = o->light_sampler; p.rr_sampler = o->rr_sampler;
    p.shader = o->shader; p.constant_value = o->constant_value;
    p.depth_min = o->depth_min; p.depth_max = o->depth_max;
    p.seed = o->seed; p.spp_offset = o->spp_offset;
    p.strata = o->spp;
    p.bitmap = bitmap;
    p.accum = (float4 *)accum;
    p.inv_w = 1.0f / (float)o->width;
    p.inv_h = 1.0f / (float)o->height;
    p.pw = 0.5f / (float)o->width;
    p.ph = 0.5f / (float)o->height;
    p.depth_point = V3{o->depth_point[0], o->depth_point[1], o->depth_point[2]};
    p.tasks = nullptr;
    p.n_tasks = o->width * 16u * bsy;
    uint32_t *counters = reinterpret_cast<uint32_t *>(scratch + kNaCounters);
    const int accel = s->opts.accelerator, mode = s->opts.bvh_mode;
    const int grid = ctx->sm_count * 16;
    uint64_t rays_closest = 0, rays_shadow = 0;
    uint32_t launches = 0;
    s->progress.store(0);
    cudaEventRecord(ctx->ev0, q);
    if (direct_shader(o->shader)) {
        launches = 1;
        if (accel == MRT_ACCEL_BVH && mode == MRT_BVH_FAST) {
            const uint32_t tiles_x = o->width / 2u;   // width is a multiple of 16, rows of 16
            cudaMemsetAsync(counters, 0, sizeof(uint32_t), q);
            k_render_noshadows_fast<<<ctx->sm_count * kNsBlocksPerSm, 128, 0, q>>>(s->dev, p, 0u, p.n_tasks, counters, tiles_x);
        } else {
            MRT_DISPATCH(launch_noshadows, accel, mode, s->dev, p, 0u, p.n_tasks, grid, q);
        }
        rays_closest = (uint64_t)p.n_tasks * o->spp;
    } else {
        const int levels = std::max(1, o->depth_max + 1);
        WaveState w{};
        w.rays = reinterpret_cast<RayRec *>(scratch + kNaRays);
        w.nodes = reinterpret_cast<NodeRec *>(scratch + kNaNodes);
        w.shadows = reinterpret_cast<ShadowRec *>(scratch + kNaShadows);
        w.levels = reinterpret_cast<Level *>(scratch + kNaLevels);
        w.root_rgb = reinterpret_cast<float4 *>(scratch + kNaRoot);
        w.counters = reinterpret_cast<unsigned long long *>(scratch + kNaWaveCounters);
        w.ray_cap = (uint32_t)std::min<size_t>(kNaRayCap, (size_t)kNoAllocWave * (levels + 2));
        w.shadow_cap = (uint32_t)std::min<size_t>(kNaShadowCap, (size_t)kNoAllocWave * o->spl * 2);
        cudaMemsetAsync(w.counters, 0, 16, q);
        const uint64_t total_roots = (uint64_t)p.n_tasks * o->spp;
        p.task_base = 0;
        uint64_t waves_issued = 0;
        uint64_t done_samples[2] = {0, 0};
        for (uint64_t r0 = 0; r0 < total_roots; r0 += kNoAllocWave) {
            if (waves_issued >= 2) {   // at most one wave queued ahead of the running one
                const int slot = (int)(waves_issued % 2);
                st = cuda_status(ctx, cudaEventSynchronize(ctx->wave_ev[slot]), "render");
                if (st != MRT_OK) return st;
                s->progress.store((uint32_t)done_samples[slot]);
            }
            if (s->stop.load()) return cancelled(ctx, q);
            w.root_first = (uint32_t)r0;
            w.n_roots = (uint32_t)std::min<uint64_t>(kNoAllocWave, total_roots - r0);
            cudaMemsetAsync(w.levels, 0, sizeof(Level) * (levels + 2), q);
            cudaMemsetAsync(counters, 0, sizeof(uint32_t) * 2 * (levels + 1), q);
            k_wave_raygen<<<grid, 128, 0, q>>>(p, w);
            for (int b = 0; b < levels; ++b) MRT_DISPATCH(launch_wave_level, accel, mode, s->dev, p, w, b, grid, q, counters);
            for (int b = levels - 1; b >= 0; --b) k_wave_resolve<<<grid, 128, 0, q>>>(s->dev, p, w, b);
            k_wave_accumulate<<<grid, 128, 0, q>>>(p, w);
            launches += 2u + 4u * (uint32_t)levels;
            const int slot = (int)(waves_issued % 2);
            cudaEventRecord(ctx->wave_ev[slot], q);
            done_samples[slot] = (r0 + w.n_roots) / std::max<uint64_t>(1, p.n_tasks);
            ++waves_issued;
        }
        unsigned long long cnt[2] = {0, 0};
        st = cuda_status(ctx, cudaMemcpyAsync(cnt, w.counters, 16, cudaMemcpyDeviceToHost, q), "counters");
        if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "render");
        rays_closest = cnt[0];
        rays_shadow = cnt[1];
    }
    cudaEventRecord(ctx->ev1, q);
    if (st == MRT_OK) st = cuda_status(ctx, cudaGetLastError(), "render kernels");
    if (st == MRT_OK) st = cuda_status(ctx, cudaEventSynchronize(ctx->ev1), "render");
    if (st == MRT_OK) st = check_kernel_error(ctx);
    s->progress.store(o->spp);
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->rays_closest = rays_closest;
        stats->rays_shadow = rays_shadow;
        stats->paths = (uint64_t)p.n_tasks * o->spp;
        stats->device_ms = ms;
        stats->trace_ms = 0.0f;
        stats->kernel_launches = launches;
        stats->reserved = 0;
    }
    return st;
}
