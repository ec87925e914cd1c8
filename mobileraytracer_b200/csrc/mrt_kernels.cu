// mrt_kernels.cu - batch traversal kernels behind mrt_trace_closest / mrt_trace_any /
// mrt_trace_closest_counts.  One thread per ray; rays are 32-byte MrtRay records read as two
// 128-bit loads.
#include "mrt_gridwalk.cuh"
#include "mrt_internal.h"

using namespace mrt;
using namespace mrt_host;

namespace {

__device__ __forceinline__ Ray load_ray(const MrtRay *rays, uint32_t i) {
    const float4 *p = reinterpret_cast<const float4 *>(rays) + 2 * (size_t)i;
    const float4 a = __ldg(p), b = __ldg(p + 1);
    Ray r;
    r.o = V3{a.x, a.y, a.z};
    r.d = V3{a.w, b.x, b.y};
    r.depth = __float_as_int(b.z);
    r.exclude = __float_as_uint(b.w);
    return r;
}

template <int ACCEL, int MODE>
__global__ void __launch_bounds__(128) k_trace_closest(DevScene s, const MrtRay *rays, uint32_t n, MrtHit *hits) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Ray r = load_ray(rays, i);
        float len;
        uint32_t id;
        const bool hit = scene_closest<ACCEL, MODE>(s, r, len, id);
        MrtHit h;
        h.t = hit ? len : kRayLengthMax;
        h.id = hit ? id : MRT_HIT_NONE;
        reinterpret_cast<uint2 *>(hits)[i] = make_uint2(__float_as_uint(h.t), h.id);
    }
}

template <int ACCEL, int MODE>
__global__ void __launch_bounds__(128) k_trace_any(DevScene s, const MrtRay *rays, const float *dist, uint32_t n,
                                                   uint8_t *occ) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Ray r = load_ray(rays, i);
        occ[i] = scene_occ<ACCEL, MODE>(s, r, dist[i]) ? 1 : 0;
    }
}

// persistent FAST-BVH versions: work items are rays of the input array
struct TraceLane {
    uint32_t i;
};
template <bool kCount>
struct TraceWork {
    const MrtRay *rays;
    MrtHit *hits;
    uint32_t *nodes, *tris;
    uint32_t n;
    uint32_t *ctr;
    __device__ uint32_t total() const { return n; }
    __device__ uint32_t *counter() const { return ctr; }
    template <class L>
    __device__ const DevScene &scene(const L &, const DevScene &s) const { return s; }
    template <class L>
    __device__ const DevScene &view(const L &, const DevScene &s) const { return s; }
    __device__ bool begin(uint32_t item, TraceLane &lane, Ray &r) const {
        lane.i = item;
        r = load_ray(rays, item);
        return true;
    }
    __device__ bool finish(TraceLane &lane, Ray &, bool hit, float t, uint32_t id, const FastTrav &tr) const {
        if (kCount) {
            nodes[lane.i] = tr.c_nodes;
            tris[lane.i] = tr.c_tris;
        } else {
            reinterpret_cast<uint2 *>(hits)[lane.i] =
                make_uint2(__float_as_uint(hit ? t : kRayLengthMax), hit ? id : MRT_HIT_NONE);
        }
        return false;
    }
};

struct AnyWork {
    const MrtRay *rays;
    const float *dist;
    uint8_t *occ;
    uint32_t n;
    uint32_t *ctr;
    __device__ uint32_t total() const { return n; }
    __device__ uint32_t *counter() const { return ctr; }
    template <class L>
    __device__ const DevScene &scene(const L &, const DevScene &s) const { return s; }
    template <class L>
    __device__ const DevScene &view(const L &, const DevScene &s) const { return s; }
    __device__ bool begin(uint32_t item, TraceLane &lane, Ray &r, float &d) const {
        lane.i = item;
        r = load_ray(rays, item);
        d = dist[item];
        return true;
    }
    __device__ void finish(TraceLane &lane, bool occluded) const { occ[lane.i] = occluded ? 1 : 0; }
};

__global__ void __launch_bounds__(128, 8) k_trace_any_persistent(DevScene s, AnyWork work) {
    TraceLane lane;
    persistent_any(s, work, lane);
}

template <bool kCount>
__global__ void __launch_bounds__(128, 8) k_trace_persistent(DevScene s, TraceWork<kCount> work) {
    TraceLane lane;
    persistent_closest<kCount>(s, work, lane);
}

__global__ void __launch_bounds__(128, kGridBlocksPerSm) k_trace_grid_persistent(DevScene s, TraceWork<false> work) {
    TraceLane lane;
    persistent_grid_closest(s, work, lane);
}

// counting replay of the grid closest hit: planes and spheres in order, then the triangle grid
// (counted: cells visited and triangle references tested), as k_trace_closest
__global__ void __launch_bounds__(128) k_trace_counts_grid(DevScene s, const MrtRay *rays, uint32_t n, uint32_t *cells,
                                                           uint32_t *refs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Ray r = load_ray(rays, i);
        float len = kRayLengthMax;
        uint32_t id = MRT_HIT_NONE;
        grid_trace<kPlane>(s, r, len, id);
        grid_trace<kSphere>(s, r, len, id);
        GridCounts c{0, 0};
        grid_trace<kTriangle, true>(s, r, len, id, &c);
        cells[i] = c.cells;
        refs[i] = c.refs;
    }
}

template <int ACCEL, int MODE>
void launch_closest(const DevScene &s, const MrtRay *rays, uint32_t n, MrtHit *hits, int grid, cudaStream_t q) {
    k_trace_closest<ACCEL, MODE><<<grid, 128, 0, q>>>(s, rays, n, hits);
}
template <int ACCEL, int MODE>
void launch_any(const DevScene &s, const MrtRay *rays, const float *dist, uint32_t n, uint8_t *occ, int grid, cudaStream_t q) {
    k_trace_any<ACCEL, MODE><<<grid, 128, 0, q>>>(s, rays, dist, n, occ);
}

#define MRT_DISPATCH(fn, accel, mode, ...)                                                                 \
    do {                                                                                                    \
        if ((accel) == MRT_ACCEL_NAIVE) fn<MRT_ACCEL_NAIVE, MRT_BVH_FAST>(__VA_ARGS__);                     \
        else if ((accel) == MRT_ACCEL_REGULAR_GRID) fn<MRT_ACCEL_REGULAR_GRID, MRT_BVH_FAST>(__VA_ARGS__);  \
        else if ((mode) == MRT_BVH_REFERENCE) fn<MRT_ACCEL_BVH, MRT_BVH_REFERENCE>(__VA_ARGS__);            \
        else fn<MRT_ACCEL_BVH, MRT_BVH_FAST>(__VA_ARGS__);                                                  \
    } while (0)

int grid_for(const MrtContext *ctx, uint32_t n) {
    const uint32_t want = (n + 127) / 128;
    const uint32_t cap = (uint32_t)ctx->sm_count * 16u;
    return (int)(want < cap ? (want ? want : 1) : cap);
}

}  // namespace

namespace mrt_host {

int persistent_grid(const MrtContext *ctx, uint32_t n) {
    const uint32_t want = (n + 127) / 128;
    const uint32_t cap = (uint32_t)ctx->sm_count * 8u;
    return (int)(want < cap ? (want ? want : 1) : cap);
}

int launch_trace_closest(MrtScene *s, const MrtRay *d_rays, uint32_t n, MrtHit *d_hits) {
    MrtContext *ctx = s->ctx;
    if (s->opts.accelerator == MRT_ACCEL_BVH && s->opts.bvh_mode == MRT_BVH_FAST) {
        cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t), ctx->stream);
        TraceWork<false> w{d_rays, d_hits, nullptr, nullptr, n, ctx->d_counters};
        k_trace_persistent<false><<<persistent_grid(ctx, n), 128, 0, ctx->stream>>>(s->dev, w);
        return cuda_status(ctx, cudaGetLastError(), "k_trace_persistent");
    }
    if (s->opts.accelerator == MRT_ACCEL_REGULAR_GRID) {
        cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t), ctx->stream);
        TraceWork<false> w{d_rays, d_hits, nullptr, nullptr, n, ctx->d_counters};
        k_trace_grid_persistent<<<persistent_grid(ctx, n), 128, 0, ctx->stream>>>(s->dev, w);
        return cuda_status(ctx, cudaGetLastError(), "k_trace_grid_persistent");
    }
    MRT_DISPATCH(launch_closest, s->opts.accelerator, s->opts.bvh_mode, s->dev, d_rays, n, d_hits, grid_for(ctx, n), ctx->stream);
    return cuda_status(ctx, cudaGetLastError(), "k_trace_closest");
}

int launch_trace_any(MrtScene *s, const MrtRay *d_rays, const float *d_dist, uint32_t n, uint8_t *d_occ) {
    MrtContext *ctx = s->ctx;
    if (s->opts.accelerator == MRT_ACCEL_BVH && s->opts.bvh_mode == MRT_BVH_FAST) {
        cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t), ctx->stream);
        AnyWork w{d_rays, d_dist, d_occ, n, ctx->d_counters};
        k_trace_any_persistent<<<persistent_grid(ctx, n), 128, 0, ctx->stream>>>(s->dev, w);
        return cuda_status(ctx, cudaGetLastError(), "k_trace_any_persistent");
    }
    MRT_DISPATCH(launch_any, s->opts.accelerator, s->opts.bvh_mode, s->dev, d_rays, d_dist, n, d_occ, grid_for(ctx, n), ctx->stream);
    return cuda_status(ctx, cudaGetLastError(), "k_trace_any");
}

int launch_trace_counts(MrtScene *s, const MrtRay *d_rays, uint32_t n, uint32_t *d_nodes, uint32_t *d_tris) {
    MrtContext *ctx = s->ctx;
    if (s->opts.accelerator == MRT_ACCEL_REGULAR_GRID) {
        k_trace_counts_grid<<<grid_for(ctx, n), 128, 0, ctx->stream>>>(s->dev, d_rays, n, d_nodes, d_tris);
        return cuda_status(ctx, cudaGetLastError(), "k_trace_counts_grid");
    }
    // the same persistent traversal as the render and trace kernels, counting its fetches
    cudaMemsetAsync(ctx->d_counters, 0, sizeof(uint32_t), ctx->stream);
    TraceWork<true> w{d_rays, nullptr, d_nodes, d_tris, n, ctx->d_counters};
    k_trace_persistent<true><<<persistent_grid(ctx, n), 128, 0, ctx->stream>>>(s->dev, w);
    return cuda_status(ctx, cudaGetLastError(), "k_trace_persistent<count>");
}

}  // namespace mrt_host
