// mrt_batch.cu - many renders as one stream of waves over a common ray pool.
//
// The reference renders one frame per Renderer::renderFrame call (Renderer.cpp:31-116); a serving
// process with many small jobs would pay a full launch sequence and a host round trip per frame and
// leave most of the GPU idle on the small ones.  Here every submitted job (scene, camera, options,
// bitmap) gets a slot in a device job table, and the host cuts the jobs' camera paths into waves:
// by default each wave is filled with the jobs that have the fewest paths left, so a small job
// finishes within a wave or two of its arrival however large the jobs queued beside it are, and a
// wave reads the trees of only a few scenes (FIFO and equal-share orders are options).
//
// A wave runs the same per-ray arithmetic as the single render (mrt_wave.cuh): camera rays, then per
// bounce level extend (persistent FAST-BVH closest hit, each lane in its own job's tree), shade
// (node record, continuation rays and shadow rays compacted with warp ballots), shadow (persistent
// any-hit); then the bottom-up resolve and the fold into each job's bitmap in sample order.  The
// kernels read the wave's description (segments of job paths) from device memory, so one CUDA graph
// captured per launch shape serves every wave; the host only copies the description and replays
// the graph.  Block size, blocks per SM and wave size come from an autotuner that times candidate
// settings on dry runs of the first wave (all the work but the fold into the bitmaps).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "mrt_internal.h"
#include "mrt_paths.cuh"

using namespace mrt;
using namespace mrt_host;

namespace {

constexpr uint32_t kMaxSegments = 256;   // jobs that contribute paths to one wave
constexpr int kRing = 8;                 // waves the host may run ahead of the device
constexpr uint32_t kMaxPipes = 4;        // waves in flight at once, each on its own stream and buffers

struct Segment {
    uint32_t job;          // job table slot
    uint32_t local_first;  // first path (task * spp + sample) of the job in this wave
    uint32_t count;
    uint32_t wave_off;     // index of the segment's first path in the wave
};

struct WaveDesc {
    uint32_t n_seg;
    uint32_t n_roots;
    uint32_t dry;          // 1: autotuner probe, nothing is written to the jobs' bitmaps
    uint32_t pad;
    Segment seg[kMaxSegments];
};

struct BatchState {
    const RenderParams *jobs;   // [max_jobs]
    const DevScene *scenes;     // [max_jobs]
    const WaveDesc *desc;
    RayRec *rays;
    NodeRec *nodes;
    ShadowRec *shadows;
    Level *levels;              // [n_levels + 2]
    float4 *root_rgb;           // [wave]
    uint32_t *root_job;         // [wave] job slot of each camera path
    uint32_t *root_local;       // [wave] path index within its job
    uint32_t ray_cap;
    uint32_t shadow_cap;
    int n_levels;
    unsigned long long *counters;   // [0] closest, [1] shadow (real waves); [2], [3] all waves
    uint32_t *work;                 // persistent work counters, 2 per level
};

__device__ __forceinline__ void path_of(const RenderParams &p, uint32_t local, Task &k, uint32_t &pixel,
                                        uint32_t &sample) {
    const uint32_t t = local / p.spp, si = local - t * p.spp;
    k = task_of(p, t);
    pixel = k.y * p.width + k.x;
    sample = p.spp_offset + si;
}

__device__ __forceinline__ Stream stream_of(const RenderParams &p, uint32_t local) {
    Task k;
    uint32_t pixel, sample;
    path_of(p, local, k, pixel, sample);
    return make_stream(p.seed, pixel, sample, p.strata, p.constant_value);
}

__global__ void k_batch_begin(BatchState b) {
    for (int i = threadIdx.x; i < b.n_levels + 2; i += blockDim.x) b.levels[i] = Level{0, 0, 0, 0};
    for (int i = threadIdx.x; i < 2 * (b.n_levels + 1); i += blockDim.x) b.work[i] = 0;
}

__global__ void k_batch_raygen(BatchState b) {
    const uint32_t n = b.desc->n_roots, n_seg = b.desc->n_seg;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n_seg;   // last segment with wave_off <= i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (b.desc->seg[mid].wave_off <= i) lo = mid; else hi = mid;
        }
        const Segment sg = b.desc->seg[lo];
        const uint32_t local = sg.local_first + (i - sg.wave_off);
        const RenderParams &p = b.jobs[sg.job];
        Task k;
        uint32_t pixel, sample;
        path_of(p, local, k, pixel, sample);
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
        b.rays[i] = rr;
        b.root_job[i] = sg.job;
        b.root_local[i] = local;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) b.levels[0] = Level{0, n, 0, 0};
}

struct BatchLane {
    uint32_t idx;
    uint32_t job;
    FastView v;   // the job scene's tree, in registers for the node and leaf steps
};

struct BatchExtendWork {
    BatchState b;
    Level L;
    uint32_t *ctr;
    __device__ uint32_t total() const { return L.count; }
    __device__ uint32_t *counter() const { return ctr; }
    __device__ const DevScene &scene(const BatchLane &lane, const DevScene &) const { return b.scenes[lane.job]; }
    __device__ const FastView &view(const BatchLane &lane, const DevScene &) const { return lane.v; }
    __device__ bool begin(uint32_t item, BatchLane &lane, Ray &r) const {
        lane.idx = L.start + item;
        const RayRec rr = b.rays[lane.idx];
        lane.job = b.root_job[rr.root];
        lane.v = fast_view(b.scenes[lane.job]);
        r = ray_of(rr);
        return true;
    }
    __device__ bool finish(BatchLane &lane, Ray &, bool hit, float t, uint32_t id, const FastTrav &) const {
        b.nodes[lane.idx].hit_t = t;
        b.nodes[lane.idx].hit_id = hit ? id : MRT_HIT_NONE;
        return false;
    }
};

struct BatchShadowWork {
    BatchState b;
    uint32_t n;
    uint32_t *ctr;
    __device__ uint32_t total() const { return n; }
    __device__ uint32_t *counter() const { return ctr; }
    __device__ const DevScene &scene(const BatchLane &lane, const DevScene &) const { return b.scenes[lane.job]; }
    __device__ const FastView &view(const BatchLane &lane, const DevScene &) const { return lane.v; }
    __device__ bool begin(uint32_t item, BatchLane &lane, Ray &r, float &dist) const {
        const ShadowRec sr = b.shadows[item];
        lane.idx = item;
        lane.job = b.root_job[b.rays[sr.node].root];
        lane.v = fast_view(b.scenes[lane.job]);
        r.o = V3{sr.ox, sr.oy, sr.oz};
        r.d = V3{sr.dx, sr.dy, sr.dz};
        r.depth = 0;
        r.exclude = sr.exclude;
        dist = sr.dist;
        return true;
    }
    __device__ void finish(BatchLane &lane, bool occluded) const {
        if (occluded) {
            const ShadowRec &sr = b.shadows[lane.idx];
            atomicOr(&b.nodes[sr.node].occluded, 1u << (sr.j & 31u));
        }
    }
};

// whole camera paths in one persistent launch (mrt_paths.cuh): work item = the wave's path i
struct BatchPathWork {
    BatchState b;
    uint32_t *ctr;
    __device__ uint32_t total() const { return b.desc->n_roots; }
    __device__ uint32_t *counter() const { return ctr; }
    __device__ const DevScene &scene(const PathLane &L) const { return b.scenes[L.job]; }
    __device__ const FastView &view(const PathLane &L) const { return L.v; }
    __device__ const RenderParams &params(const PathLane &L) const { return b.jobs[L.job]; }
    __device__ void begin(uint32_t i, PathLane &L, Ray &r) const {
        const uint32_t n_seg = b.desc->n_seg;
        uint32_t lo = 0, hi = n_seg;   // last segment with wave_off <= i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (b.desc->seg[mid].wave_off <= i) lo = mid; else hi = mid;
        }
        const Segment sg = b.desc->seg[lo];
        const uint32_t local = sg.local_first + (i - sg.wave_off);
        const RenderParams &p = b.jobs[sg.job];
        Task k;
        uint32_t pixel, sample;
        path_of(p, local, k, pixel, sample);
        L.st = make_stream(p.seed, pixel, sample, p.strata, p.constant_value);
        r = primary_ray(p, k, L.st);
        L.item = i;
        L.job = sg.job;
        L.v = fast_view(b.scenes[sg.job]);
        L.top = 1;
        L.fr[0].code = 1u;
        L.fr[0].depth = 1;
        L.fr[0].slot = 0;
        b.root_job[i] = sg.job;
        b.root_local[i] = local;
    }
    __device__ void deliver(const PathLane &L, V3 rgb, bool flag) const {
        b.root_rgb[L.item] = make_float4(rgb.x, rgb.y, rgb.z, flag ? 1.0f : 0.0f);
    }
    __device__ void count(uint32_t n_closest, uint32_t n_shadow) const {
        const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, n_closest), d = __reduce_add_sync(0xFFFFFFFFu, n_shadow);
        if ((threadIdx.x & 31) == 0) {
            if (!b.desc->dry) {
                atomicAdd(&b.counters[0], (unsigned long long)c);
                atomicAdd(&b.counters[1], (unsigned long long)d);
            }
            atomicAdd(&b.counters[2], (unsigned long long)c);
            atomicAdd(&b.counters[3], (unsigned long long)d);
        }
    }
};

__global__ void __launch_bounds__(128, 8) k_batch_paths(BatchState b) {
    BatchPathWork work{b, b.work};
    persistent_paths(work);
}

// threads per SM the batch's traversal kernels are compiled for (registers per thread: 65536 / this);
// the 256-job batch: 1030 Mrays/s at 768, 1024 at 896, 998 at 1024 (spills at 64 registers)
#ifndef MRT_BATCH_THREADS_PER_SM
#define MRT_BATCH_THREADS_PER_SM 768
#endif
constexpr int kBatchThreadsPerSm = MRT_BATCH_THREADS_PER_SM;

template <int kBlock, int Q>
__global__ void __launch_bounds__(kBlock, kBatchThreadsPerSm / kBlock) k_batch_extend(BatchState b, int level) {
    Level L = b.levels[level];
    L.start = min(L.start, b.ray_cap);
    L.count = min(L.count, b.ray_cap - L.start);
    BatchExtendWork work{b, L, b.work + 2 * level};
    BatchLane lane;
    persistent_closest<false, Q>(b.scenes[0], work, lane);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (!b.desc->dry) atomicAdd(&b.counters[0], (unsigned long long)L.count);
        atomicAdd(&b.counters[2], (unsigned long long)L.count);
    }
}

template <int kBlock>
__global__ void __launch_bounds__(kBlock, kBatchThreadsPerSm / kBlock) k_batch_shadow(BatchState b, int level) {
    const uint32_t n = min(b.levels[level].shadow_count, b.shadow_cap);
    BatchShadowWork work{b, n, b.work + 2 * level + 1};
    BatchLane lane;
    persistent_any(b.scenes[0], work, lane);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (!b.desc->dry) atomicAdd(&b.counters[1], (unsigned long long)n);
        atomicAdd(&b.counters[3], (unsigned long long)n);
    }
}

// NoShadows / DepthMap / DiffuseMaterial (NoShadows.cpp:19-65, DepthMap.cpp:19-26,
// DiffuseMaterial.cpp:16-38) in node form: the value is final at the camera ray
__device__ __forceinline__ void shade_direct_node(const DevScene &s, const RenderParams &p, const RayRec &rr,
                                                     uint32_t hit_id, float hit_t, const Stream &st, ShadeLane &o) {
    o.n_child = 0;
    o.child_mask = 0;
    o.n_shadow = 0;
    o.shaded = false;
    NodeRec &nd = o.nd;
    nd.flags = kMiss;
    nd.occluded = 0;
    nd.child_flag = 0;
    nd.child[0] = nd.child[1] = nd.child[2] = V3{0, 0, 0};
    nd.kd = nd.ks = nd.kt = V3{0, 0, 0};
    nd.point = nd.normal = V3{0, 0, 0};
    nd.hit_id = hit_id;
    nd.hit_t = hit_t;
    if (hit_id == MRT_HIT_NONE) return;
    const Ray r = ray_of(rr);
    Isect it;
    if (!make_isect(s, r, hit_id, it)) return;
    nd.flags = kEmit;   // resolves to the value in `point`
    nd.point = shade_direct(s, p, st, r, it);
}

__global__ void __launch_bounds__(128) k_batch_shade(BatchState b, int level) {
    Level L = b.levels[level];
    L.start = min(L.start, b.ray_cap);
    L.count = min(L.count, b.ray_cap - L.start);
    Level *next = &b.levels[level + 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) next->start = L.start + L.count;
    const uint32_t next_start = L.start + L.count;
    const uint32_t n_iter = (L.count + blockDim.x - 1) / blockDim.x;   // whole warps iterate together
    for (uint32_t it_ = blockIdx.x; it_ < n_iter; it_ += gridDim.x) {
        const uint32_t i = it_ * blockDim.x + threadIdx.x;
        const bool active = i < L.count;
        const uint32_t idx = L.start + (active ? i : 0);
        ShadeLane o;
        o.n_child = 0;
        o.child_mask = 0;
        o.n_shadow = 0;
        o.shaded = false;
        RayRec rr;
        Stream st;
        uint32_t job = 0;
        if (active) {
            rr = b.rays[idx];
            job = b.root_job[rr.root];
            const RenderParams &p = b.jobs[job];
            const DevScene &s = b.scenes[job];
            st = stream_of(p, b.root_local[rr.root]);
            const NodeRec &in = b.nodes[idx];
            if (direct_shader(p.shader)) shade_direct_node(s, p, rr, in.hit_id, in.hit_t, st, o);
            else shade_ray(s, p, rr, in.hit_id, in.hit_t, st, o);
            store_node(b.nodes[idx], o.nd);
        }
        const uint32_t cbase = warp_alloc(o.n_child, &next->count);
        const uint32_t sbase = warp_alloc(o.n_shadow, &b.levels[level].shadow_count);
        if (!active) continue;
        const DevScene &s = b.scenes[job];
        emit_children(s, o, rr, st, idx, next_start + cbase, b.rays, b.ray_cap);
        emit_shadows(s, b.jobs[job], st, o, rr, idx, sbase, b.shadows, b.shadow_cap);
    }
}

__global__ void __launch_bounds__(128) k_batch_resolve(BatchState b, int level) {
    Level L = b.levels[level];
    L.start = min(L.start, b.ray_cap);
    L.count = min(L.count, b.ray_cap - L.start);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.count; i += gridDim.x * blockDim.x) {
        const uint32_t idx = L.start + i;
        const NodeRec &nd = b.nodes[idx];
        const RayRec &rr = b.rays[idx];
        V3 rgb{0.0f, 0.0f, 0.0f};
        bool flag = false;
        const uint32_t kind = nd.flags & 3u;
        if (kind == kEmit) {
            rgb = nd.point;
            flag = true;
        } else if (kind == kShaded) {   // misses and cut nodes are black
            const uint32_t job = b.root_job[rr.root];
            const RenderParams &p = b.jobs[job];
            const Stream st = stream_of(p, b.root_local[rr.root]);
            resolve_node(b.scenes[job], p, nd, rr, st, rgb, flag);
        }
        if (rr.parent == 0xFFFFFFFFu) {
            b.root_rgb[rr.root] = make_float4(rgb.x, rgb.y, rgb.z, flag ? 1.0f : 0.0f);
        } else {
            NodeRec &pn = b.nodes[rr.parent];
            pn.child[rr.slot] = rgb;
            if (flag) atomicOr(&pn.child_flag, 1u << rr.slot);
        }
    }
}

// fold each pixel's samples of this wave into its bitmap in sample order (Renderer.cpp:105-107): the
// thread of the pixel's first sample in the wave folds all of them
__global__ void k_batch_accumulate(BatchState b) {
    if (b.desc->dry) return;
    const uint32_t n = b.desc->n_roots;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t job = b.root_job[i], local = b.root_local[i];
        const RenderParams &p = b.jobs[job];
        const uint32_t t = local / p.spp;
        if (i > 0 && b.root_job[i - 1] == job && b.root_local[i - 1] / p.spp == t) continue;
        const Task k = task_of(p, t);
        const int64_t slot = p.accum ? accum_slot(p, k) : -1;
        uint32_t bm = p.bitmap[k.index];
        float4 acc = slot >= 0 ? p.accum[slot] : make_float4(0, 0, 0, 0);
        for (uint32_t g = i; g < n && b.root_job[g] == job; ++g) {
            const uint32_t lg = b.root_local[g];
            if (lg / p.spp != t) break;
            const float4 c = b.root_rgb[g];
            const V3 rgb{c.x, c.y, c.z};
            const uint32_t sample = p.spp_offset + (lg - t * p.spp);
            bm = incremental_avg(rgb, bm, sample + 1u);
            acc.x += rgb.x; acc.y += rgb.y; acc.z += rgb.z; acc.w += 1.0f;
        }
        p.bitmap[k.index] = bm;
        if (slot >= 0) p.accum[slot] = acc;
    }
}

bool plain_rectangle(const MrtRenderOpts &o, uint32_t stride_bytes) {
    if (o.width < 16 || o.height < 16) return false;
    const uint32_t bsy = o.height / 16u;
    return o.width % 16u == 0 && stride_bytes == 4u * o.width && o.height / bsy == 16u;
}

}  // namespace

struct BatchPipe {
    cudaStream_t stream = nullptr;
    DevBuf d_desc, d_rays, d_nodes, d_shadows, d_levels, d_root_rgb, d_root_job, d_root_local, d_work;
    std::map<std::pair<uint32_t, uint32_t>, cudaGraphExec_t> graphs;   // per (block threads, blocks per SM)
    uint64_t jobs_seen = 0;      // job uploads this pipeline's stream has waited for
};

struct MrtBatch {
    MrtContext *ctx = nullptr;
    MrtBatchOpts opts{};
    uint32_t max_jobs = 4096;
    int n_levels = 9;
    uint32_t wave_cap = 0;           // largest wave the buffers hold
    uint32_t n_pipes_alloc = 1;      // pipelines with buffers
    // settings in use
    uint32_t wave_roots = 0, block_threads = 0, blocks_per_sm = 0, n_pipes = 1;
    bool tuned = false;
    uint32_t autotuned = 0;
    // device
    DevBuf d_jobs, d_scenes, d_counters;
    BatchPipe pipes[kMaxPipes];
    // pinned host mirrors
    RenderParams *h_jobs = nullptr;
    DevScene *h_scenes = nullptr;
    WaveDesc *h_desc = nullptr;      // [kRing]
    // jobs (host view)
    struct Job {
        uint64_t id = 0;
        uint64_t total = 0;          // paths
        uint64_t next = 0;           // next path to schedule
        bool live = false;
    };
    std::vector<Job> slots;          // [max_jobs], slot = id % max_jobs
    std::vector<uint32_t> active;    // slots with paths left, submission order
    uint64_t next_id = 0;
    uint64_t jobs_done = 0;
    uint64_t jobs_uploaded = 0;      // submissions whose table rows are queued on ctx->stream
    cudaEvent_t ev_jobs = nullptr;   // recorded after the latest job upload
    std::vector<uint64_t> newly_done;
    std::map<int64_t, std::vector<uint32_t>> finishing;   // wave -> slots whose last paths it runs
    // waves: ring slot r = wave % kRing
    int64_t waves_launched = 0, waves_done = 0;
    cudaEvent_t ev_start[kRing] = {}, ev_end[kRing] = {}, ev_acc[kRing] = {};
    cudaEvent_t ev_first = nullptr;  // start of the current busy period
    float period_ms = 0.0f;          // latest wave end seen in the current busy period
    uint64_t paths = 0;
    uint64_t waves_paths = 0;        // waves run as whole-path launches
    double busy_ms = 0.0;
    unsigned long long counters_host[4] = {0, 0, 0, 0};
};

namespace {

BatchState state_of(MrtBatch *b, int pipe) {
    const BatchPipe &P = b->pipes[pipe];
    BatchState s{};
    s.jobs = (const RenderParams *)b->d_jobs.ptr;
    s.scenes = (const DevScene *)b->d_scenes.ptr;
    s.desc = (const WaveDesc *)P.d_desc.ptr;
    s.rays = (RayRec *)P.d_rays.ptr;
    s.nodes = (NodeRec *)P.d_nodes.ptr;
    s.shadows = (ShadowRec *)P.d_shadows.ptr;
    s.levels = (Level *)P.d_levels.ptr;
    s.root_rgb = (float4 *)P.d_root_rgb.ptr;
    s.root_job = (uint32_t *)P.d_root_job.ptr;
    s.root_local = (uint32_t *)P.d_root_local.ptr;
    s.ray_cap = (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, (uint64_t)b->wave_cap * (b->n_levels + 2));
    s.shadow_cap = (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, (uint64_t)b->wave_cap *
                                                                   std::max(1u, b->opts.max_spl) * 2ull);
    s.n_levels = b->n_levels;
    s.counters = (unsigned long long *)b->d_counters.ptr;
    s.work = (uint32_t *)P.d_work.ptr;
    return s;
}

template <int kBlock>
void launch_traversal(const BatchState &s, int level, int grid, cudaStream_t q, bool extend) {
    if (extend) k_batch_extend<kBlock, kNodeQuorum><<<grid, kBlock, 0, q>>>(s, level);
    else k_batch_shadow<kBlock><<<grid, kBlock, 0, q>>>(s, level);
}

// the wave up to the per-sample values: camera rays, every bounce level, the bottom-up resolve
// (threads = 0: whole paths in one persistent launch instead)
void launch_trace_kernels(MrtBatch *b, int pipe, uint32_t threads, uint32_t bps, cudaStream_t q) {
    const BatchState s = state_of(b, pipe);
    const int sm = b->ctx->sm_count;
    const int tgrid = sm * (int)bps;
    const int grid = sm * 16;
    if (threads == 0) {
        k_batch_begin<<<1, 64, 0, q>>>(s);
        k_batch_paths<<<sm * 8, 128, 0, q>>>(s);
        return;
    }
    auto trav = [&](int level, bool extend) {
        if (threads == 64) launch_traversal<64>(s, level, tgrid, q, extend);
        else if (threads == 256) launch_traversal<256>(s, level, tgrid, q, extend);
        else launch_traversal<128>(s, level, tgrid, q, extend);
    };
    k_batch_begin<<<1, 64, 0, q>>>(s);
    k_batch_raygen<<<grid, 128, 0, q>>>(s);
    for (int l = 0; l < b->n_levels; ++l) {
        trav(l, true);
        k_batch_shade<<<grid, 128, 0, q>>>(s, l);
        trav(l, false);
    }
    for (int l = b->n_levels - 1; l >= 0; --l) k_batch_resolve<<<grid, 128, 0, q>>>(s, l);
}

int trace_graph(MrtBatch *b, int pipe, uint32_t threads, uint32_t bps, cudaGraphExec_t *out) {
    BatchPipe &P = b->pipes[pipe];
    auto key = std::make_pair(threads, bps);
    auto it = P.graphs.find(key);
    if (it != P.graphs.end()) { *out = it->second; return MRT_OK; }
    MrtContext *ctx = b->ctx;
    cudaGraph_t g = nullptr;
    int st = cuda_status(ctx, cudaStreamBeginCapture(P.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    if (st != MRT_OK) return st;
    launch_trace_kernels(b, pipe, threads, bps, P.stream);
    st = cuda_status(ctx, cudaStreamEndCapture(P.stream, &g), "end capture");
    if (st != MRT_OK) return st;
    cudaGraphExec_t exec = nullptr;
    st = cuda_status(ctx, cudaGraphInstantiate(&exec, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    if (st != MRT_OK) return st;
    P.graphs[key] = exec;
    *out = exec;
    return MRT_OK;
}

// fill the wave description from the jobs with paths left, by the batch's policy:
//   SMALLEST_FIRST  jobs with the fewest paths left first (a small job completes in the next wave
//                   however much work is queued), ties in submission order;
//   FIFO            submission order;
//   EQUAL_SHARE     an equal share for each of the first kMaxSegments jobs, leftovers to the
//                   earliest (every job advances every wave; waves touch many scenes).
// The first two fill a wave from as few jobs as possible, so the scenes a wave reads stay few.
uint32_t plan_wave(MrtBatch *b, WaveDesc &d, uint32_t wave, bool commit, int64_t wave_index, uint32_t policy) {
    d.n_seg = 0;
    d.n_roots = 0;
    d.dry = commit ? 0u : 1u;
    if (b->active.empty()) return 0;
    std::vector<uint32_t> order(b->active);
    if (policy == MRT_BATCH_SMALLEST_FIRST)
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
            return b->slots[x].total - b->slots[x].next < b->slots[y].total - b->slots[y].next;
        });
    const size_t n_act = std::min<size_t>(order.size(), kMaxSegments);
    std::vector<uint64_t> take(n_act, 0);
    uint64_t room = wave;
    if (policy == MRT_BATCH_EQUAL_SHARE) {
        const uint64_t share = std::max<uint64_t>(1, wave / n_act);
        for (size_t a = 0; a < n_act && room; ++a) {
            const MrtBatch::Job &j = b->slots[order[a]];
            take[a] = std::min<uint64_t>({j.total - j.next, share, room});
            room -= take[a];
        }
    }
    for (size_t a = 0; a < n_act && room; ++a) {
        const MrtBatch::Job &j = b->slots[order[a]];
        const uint64_t more = std::min<uint64_t>(j.total - j.next - take[a], room);
        take[a] += more;
        room -= more;
    }
    uint32_t off = 0;
    for (size_t a = 0; a < n_act; ++a) {
        if (!take[a]) continue;
        MrtBatch::Job &j = b->slots[order[a]];
        Segment &sg = d.seg[d.n_seg++];
        sg.job = order[a];
        sg.local_first = (uint32_t)j.next;
        sg.count = (uint32_t)take[a];
        sg.wave_off = off;
        off += sg.count;
        if (commit) {
            j.next += take[a];
            if (j.next == j.total) b->finishing[wave_index].push_back(order[a]);
        }
    }
    d.n_roots = off;
    if (commit) {
        std::vector<uint32_t> keep;
        keep.reserve(b->active.size());
        for (uint32_t slot : b->active)
            if (b->slots[slot].next < b->slots[slot].total) keep.push_back(slot);
        b->active.swap(keep);
    }
    return off;
}

// Kernel of a wave when the caller left it open: whole paths per lane when no job holds half of
// the wave (a mix of small jobs: level barriers and launches dominate the wavefront there), the
// level-by-level wavefront when one job dominates (its rays are coherent level by level).
bool whole_paths_wave(const WaveDesc &d) {
    uint32_t largest = 0;
    for (uint32_t k = 0; k < d.n_seg; ++k) largest = std::max(largest, d.seg[k].count);
    return 2ull * largest < d.n_roots;
}

// one wave on pipeline `pipe`: description copy, the traced part (a graph replay), then the fold
// into the bitmaps, which waits for the previous wave's fold (a pixel's samples may straddle the
// two waves, and their order must stay the sample order)
int run_wave(MrtBatch *b, const WaveDesc &d, int pipe, uint32_t threads, uint32_t bps, int ring, int prev_ring) {
    MrtContext *ctx = b->ctx;
    BatchPipe &P = b->pipes[pipe];
    cudaStream_t q = P.stream;
    if (P.jobs_seen != b->jobs_uploaded) {
        cudaStreamWaitEvent(q, b->ev_jobs, 0);
        P.jobs_seen = b->jobs_uploaded;
    }
    if (ring >= 0) cudaEventRecord(b->ev_start[ring], q);
    const size_t bytes = offsetof(WaveDesc, seg) + sizeof(Segment) * std::max(1u, d.n_seg);
    int st = cuda_status(ctx, cudaMemcpyAsync(P.d_desc.ptr, &d, bytes, cudaMemcpyHostToDevice, q), "wave description");
    if (st != MRT_OK) return st;
    if (b->opts.no_graph) {
        launch_trace_kernels(b, pipe, threads, bps, q);
    } else {
        cudaGraphExec_t g = nullptr;
        st = trace_graph(b, pipe, threads, bps, &g);
        if (st != MRT_OK) return st;
        st = cuda_status(ctx, cudaGraphLaunch(g, q), "graph launch");
        if (st != MRT_OK) return st;
    }
    if (!d.dry) {
        if (prev_ring >= 0) cudaStreamWaitEvent(q, b->ev_acc[prev_ring], 0);
        k_batch_accumulate<<<ctx->sm_count * 16, 128, 0, q>>>(state_of(b, pipe));
        if (ring >= 0) cudaEventRecord(b->ev_acc[ring], q);
    }
    if (ring >= 0) cudaEventRecord(b->ev_end[ring], q);
    return cuda_status(ctx, cudaGetLastError(), "wave kernels");
}

// retire completed waves in launch order: jobs whose last wave finished become done
int retire(MrtBatch *b, bool wait_one) {
    while (b->waves_done < b->waves_launched) {
        const int r = (int)(b->waves_done % kRing);
        cudaError_t e = wait_one ? cudaEventSynchronize(b->ev_end[r]) : cudaEventQuery(b->ev_end[r]);
        if (e == cudaErrorNotReady) return MRT_OK;
        if (e != cudaSuccess) return cuda_status(b->ctx, e, "wave");
        wait_one = false;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, b->ev_first, b->ev_end[r]) == cudaSuccess) b->period_ms = std::max(b->period_ms, ms);
        auto it = b->finishing.find(b->waves_done);
        if (it != b->finishing.end()) {
            for (uint32_t slot : it->second) {
                b->slots[slot].live = false;
                b->newly_done.push_back(b->slots[slot].id);
                ++b->jobs_done;
            }
            b->finishing.erase(it);
        }
        ++b->waves_done;
        if (b->waves_done == b->waves_launched) {   // the device went idle: close the busy period
            b->busy_ms += b->period_ms;
            b->period_ms = 0.0f;
        }
    }
    return MRT_OK;
}

int read_counters(MrtBatch *b, unsigned long long *c) {
    MrtContext *ctx = b->ctx;
    int st = cuda_status(ctx, cudaMemcpyAsync(c, b->d_counters.ptr, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                              ctx->stream), "counters");
    if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "counters");
    return st;
}

int check_batch_error(MrtBatch *b) {
    int st = check_kernel_error(b->ctx);
    if (st != MRT_OK) return st;
    return read_counters(b, b->counters_host);
}

// time candidate settings on dry runs of the next wave's paths (the fold into the bitmaps skipped):
// the traversal launch shape, then the wave size, then how many waves run at once
int autotune(MrtBatch *b) {
    MrtContext *ctx = b->ctx;
    cudaStream_t q = ctx->stream;
    const MrtBatchOpts &o = b->opts;
    std::vector<std::pair<uint32_t, uint32_t>> shapes;
    if (o.kernel == MRT_BATCH_KERNEL_PATHS) {
        shapes.push_back({0u, 8u});
    } else if (o.block_threads && o.blocks_per_sm) {
        shapes.push_back({o.block_threads, o.blocks_per_sm});
    } else {
        const uint32_t ts[3] = {64, 128, 256};
        const uint32_t per_sm_threads[3] = {512, 1024, 2048};
        for (uint32_t t : ts) {
            if (o.block_threads && t != o.block_threads) continue;
            for (uint32_t pt : per_sm_threads) {
                const uint32_t bps = pt / t;
                if (bps < 1 || bps > 16 || (o.blocks_per_sm && bps != o.blocks_per_sm)) continue;
                shapes.push_back({t, bps});
            }
        }
    }
    std::vector<uint32_t> waves;
    if (o.wave_roots) waves.push_back(std::min(o.wave_roots, b->wave_cap));
    else for (uint32_t w = b->wave_cap; w >= (1u << 17) && waves.size() < 3; w >>= 1) waves.push_back(w);
    if (waves.empty()) waves.push_back(b->wave_cap);
    std::vector<uint32_t> pipes;
    if (o.pipelines) pipes.push_back(std::min(o.pipelines, b->n_pipes_alloc));
    else for (uint32_t p = 1; p <= b->n_pipes_alloc; ++p) pipes.push_back(p);
    b->block_threads = shapes[0].first;
    b->blocks_per_sm = shapes[0].second;
    b->wave_roots = waves[0];
    b->n_pipes = pipes[0];
    if (shapes.size() == 1 && waves.size() == 1 && pipes.size() == 1) return MRT_OK;

    cudaEvent_t e0 = nullptr, e1 = nullptr, ep[kMaxPipes] = {};
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (uint32_t p = 0; p < b->n_pipes_alloc; ++p) cudaEventCreateWithFlags(&ep[p], cudaEventDisableTiming);
    // rays per ms of `np` concurrent dry waves of w paths each
    auto probe = [&](uint32_t t, uint32_t bps, uint32_t w, uint32_t np, double &rate) -> int {
        WaveDesc &d = b->h_desc[0];
        rate = 0.0;
        // an equal share of every queued job: the probe sees the batch's mix, not only its first jobs
        if (plan_wave(b, d, w, false, -1, MRT_BATCH_EQUAL_SHARE) == 0) return MRT_OK;
        unsigned long long c0[4], c1[4];
        int st = read_counters(b, c0);
        if (st != MRT_OK) return st;
        cudaEventRecord(e0, q);
        for (uint32_t p = 0; p < np && st == MRT_OK; ++p) {
            cudaStreamWaitEvent(b->pipes[p].stream, e0, 0);
            st = run_wave(b, d, (int)p, t, bps, -1, -1);
            cudaEventRecord(ep[p], b->pipes[p].stream);
            cudaStreamWaitEvent(q, ep[p], 0);
        }
        if (st != MRT_OK) return st;
        cudaEventRecord(e1, q);
        st = cuda_status(ctx, cudaEventSynchronize(e1), "probe");
        if (st == MRT_OK) st = read_counters(b, c1);
        if (st != MRT_OK) return st;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        rate = ms > 0.0f ? ((double)(c1[2] - c0[2]) + (double)(c1[3] - c0[3])) / ms : 0.0;
        ++b->autotuned;
        return MRT_OK;
    };
    int st = MRT_OK;
    double rate = 0.0, best = -1.0;
    uint32_t bt = shapes[0].first, bb = shapes[0].second, bw = waves[waves.size() / 2], bp = pipes[0];
    st = probe(bt, bb, bw, 1, rate);   // warm-up: graphs, caches
    for (size_t i = 0; st == MRT_OK && shapes.size() > 1 && i < shapes.size(); ++i) {
        st = probe(shapes[i].first, shapes[i].second, bw, 1, rate);
        if (st == MRT_OK && rate > best) { best = rate; bt = shapes[i].first; bb = shapes[i].second; }
    }
    best = -1.0;
    for (size_t i = 0; st == MRT_OK && waves.size() > 1 && i < waves.size(); ++i) {
        st = probe(bt, bb, waves[i], 1, rate);
        if (st == MRT_OK && rate > best) { best = rate; bw = waves[i]; }
    }
    best = -1.0;
    const uint32_t w0 = bw;
    for (size_t i = 0; st == MRT_OK && pipes.size() > 1 && i < pipes.size(); ++i) {
        for (uint32_t w : {w0, std::max(1024u, w0 / 2)}) {
            if (pipes[i] == 1 && w != w0) continue;
            st = probe(bt, bb, w, pipes[i], rate);
            if (st != MRT_OK) break;
            if (rate > best) { best = rate; bp = pipes[i]; bw = w; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (uint32_t p = 0; p < b->n_pipes_alloc; ++p) cudaEventDestroy(ep[p]);
    if (st != MRT_OK) return st;
    b->block_threads = bt;
    b->blocks_per_sm = bb;
    b->wave_roots = bw;
    b->n_pipes = bp;
    return MRT_OK;
}

void free_batch(MrtBatch *b) {
    if (!b) return;
    for (uint32_t p = 0; p < kMaxPipes; ++p) {
        BatchPipe &P = b->pipes[p];
        if (P.stream) cudaStreamSynchronize(P.stream);
        for (auto &kv : P.graphs) cudaGraphExecDestroy(kv.second);
        DevBuf *bufs[] = {&P.d_desc, &P.d_rays, &P.d_nodes, &P.d_shadows, &P.d_levels, &P.d_root_rgb, &P.d_root_job,
                          &P.d_root_local, &P.d_work};
        for (DevBuf *x : bufs) dev_free(*x);
        if (P.stream) cudaStreamDestroy(P.stream);
    }
    if (b->ctx && b->ctx->stream) cudaStreamSynchronize(b->ctx->stream);
    dev_free(b->d_jobs);
    dev_free(b->d_scenes);
    dev_free(b->d_counters);
    if (b->h_jobs) cudaFreeHost(b->h_jobs);
    if (b->h_scenes) cudaFreeHost(b->h_scenes);
    if (b->h_desc) cudaFreeHost(b->h_desc);
    for (int r = 0; r < kRing; ++r) {
        if (b->ev_start[r]) cudaEventDestroy(b->ev_start[r]);
        if (b->ev_end[r]) cudaEventDestroy(b->ev_end[r]);
        if (b->ev_acc[r]) cudaEventDestroy(b->ev_acc[r]);
    }
    if (b->ev_jobs) cudaEventDestroy(b->ev_jobs);
    if (b->ev_first) cudaEventDestroy(b->ev_first);
    delete b;
}

}  // namespace

extern "C" {

int mrt_batch_create(MrtContext *ctx, const MrtBatchOpts *opts, MrtBatch **out) {
    if (!ctx || !out) return MRT_ERR_ARG;
    *out = nullptr;
    MrtBatchOpts o{};
    if (opts) o = *opts;
    if (o.kernel == MRT_BATCH_KERNEL_PATHS && o.max_depth + 1 > (uint32_t)kPathFrames) {
        set_error(ctx, "mrt_batch_create: whole-path launches hold depth_max <= %d", kPathFrames - 1);
        return MRT_ERR_ARG;
    }
    if (o.kernel > MRT_BATCH_KERNEL_PATHS) {
        set_error(ctx, "mrt_batch_create: kernel must be 0 (autotuned), MRT_BATCH_KERNEL_WAVEFRONT or MRT_BATCH_KERNEL_PATHS");
        return MRT_ERR_ARG;
    }
    if (o.block_threads && o.block_threads != 64 && o.block_threads != 128 && o.block_threads != 256) {
        set_error(ctx, "mrt_batch_create: block_threads must be 64, 128 or 256");
        return MRT_ERR_ARG;
    }
    if (o.blocks_per_sm > 16 || o.max_depth > 30 || o.max_spl > 32 || o.max_jobs > (1u << 20) ||
        o.policy > MRT_BATCH_EQUAL_SHARE || o.pipelines > kMaxPipes) {
        set_error(ctx, "mrt_batch_create: blocks_per_sm <= 16, max_depth <= 30, max_spl <= 32, max_jobs <= 2^20, "
                       "pipelines <= %d, policy one of MRT_BATCH_*", kMaxPipes);
        return MRT_ERR_ARG;
    }
    if (!o.max_jobs) o.max_jobs = 4096;
    if (!o.max_depth) o.max_depth = 8;
    if (!o.max_spl) o.max_spl = 4;
    if (!o.max_wave_roots) o.max_wave_roots = 1u << 21;
    if (o.wave_roots) o.max_wave_roots = std::max(o.max_wave_roots, o.wave_roots);
    o.max_wave_roots = std::max(1024u, std::min(o.max_wave_roots, 1u << 24));
    if (o.wave_roots) o.wave_roots = std::max(1024u, std::min(o.wave_roots, o.max_wave_roots));
    cudaSetDevice(ctx->device);
    MrtBatch *b = new MrtBatch();
    b->ctx = ctx;
    b->opts = o;
    b->max_jobs = o.max_jobs;
    b->n_levels = (int)o.max_depth + 1;
    b->wave_cap = o.max_wave_roots;
    b->n_pipes_alloc = o.pipelines ? o.pipelines : kMaxPipes;
    b->slots.resize(o.max_jobs);
    const uint64_t ray_cap = (uint64_t)b->wave_cap * (b->n_levels + 2);
    const uint64_t shadow_cap = (uint64_t)b->wave_cap * o.max_spl * 2ull;
    if (ray_cap > 0xFFFFFFF0ull || shadow_cap > 0xFFFFFFF0ull) {
        set_error(ctx, "mrt_batch_create: wave too large for the ray pool");
        delete b;
        return MRT_ERR_ARG;
    }
    int st = MRT_OK;
    auto A = [&](DevBuf &x, size_t bytes) { if (st == MRT_OK) st = dev_alloc(ctx, x, bytes); };
    A(b->d_jobs, sizeof(RenderParams) * o.max_jobs);
    A(b->d_scenes, sizeof(DevScene) * o.max_jobs);
    A(b->d_counters, 4 * sizeof(unsigned long long));
    for (uint32_t p = 0; p < b->n_pipes_alloc && st == MRT_OK; ++p) {
        BatchPipe &P = b->pipes[p];
        st = cuda_status(ctx, cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        A(P.d_desc, sizeof(WaveDesc));
        A(P.d_rays, sizeof(RayRec) * ray_cap);
        A(P.d_nodes, sizeof(NodeRec) * ray_cap);
        A(P.d_shadows, sizeof(ShadowRec) * shadow_cap);
        A(P.d_levels, sizeof(Level) * (b->n_levels + 2));
        A(P.d_root_rgb, sizeof(float4) * b->wave_cap);
        A(P.d_root_job, sizeof(uint32_t) * b->wave_cap);
        A(P.d_root_local, sizeof(uint32_t) * b->wave_cap);
        A(P.d_work, sizeof(uint32_t) * 2 * (b->n_levels + 1));
    }
    if (st == MRT_OK) st = cuda_status(ctx, cudaMallocHost(&b->h_jobs, sizeof(RenderParams) * o.max_jobs), "cudaMallocHost");
    if (st == MRT_OK) st = cuda_status(ctx, cudaMallocHost(&b->h_scenes, sizeof(DevScene) * o.max_jobs), "cudaMallocHost");
    if (st == MRT_OK) st = cuda_status(ctx, cudaMallocHost(&b->h_desc, sizeof(WaveDesc) * kRing), "cudaMallocHost");
    for (int r = 0; st == MRT_OK && r < kRing; ++r) {
        st = cuda_status(ctx, cudaEventCreate(&b->ev_start[r]), "cudaEventCreate");
        if (st == MRT_OK) st = cuda_status(ctx, cudaEventCreate(&b->ev_end[r]), "cudaEventCreate");
        if (st == MRT_OK) st = cuda_status(ctx, cudaEventCreateWithFlags(&b->ev_acc[r], cudaEventDisableTiming), "cudaEventCreate");
    }
    if (st == MRT_OK) st = cuda_status(ctx, cudaEventCreateWithFlags(&b->ev_jobs, cudaEventDisableTiming), "cudaEventCreate");
    if (st == MRT_OK) st = cuda_status(ctx, cudaEventCreate(&b->ev_first), "cudaEventCreate");
    if (st == MRT_OK) st = cuda_status(ctx, cudaMemsetAsync(b->d_counters.ptr, 0, 4 * sizeof(unsigned long long), ctx->stream), "memset");
    if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "mrt_batch_create");
    if (st != MRT_OK) { free_batch(b); return st; }
    *out = b;
    return MRT_OK;
}

void mrt_batch_destroy(MrtBatch *b) { free_batch(b); }

int mrt_batch_submit(MrtBatch *b, const MrtBatchJob *job, uint64_t *job_id) {
    if (!b || !job || !job->scene) return MRT_ERR_ARG;
    MrtContext *ctx = b->ctx;
    const MrtRenderOpts *o = &job->opts;
    MrtScene *s = job->scene;
    if (!s->built) { set_error(ctx, "mrt_batch_submit: scene not built"); return MRT_ERR_STATE; }
    if (s->ctx->device != ctx->device || s->opts.accelerator != MRT_ACCEL_BVH || s->opts.bvh_mode != MRT_BVH_FAST) {
        set_error(ctx, "mrt_batch_submit: the scene must be built with MRT_ACCEL_BVH + MRT_BVH_FAST on the batch's device");
        return MRT_ERR_ARG;
    }
    if (o->shader < MRT_SHADER_NOSHADOWS || o->shader > MRT_SHADER_DIFFUSE || o->spp == 0 ||
        (o->spl == 0 && (o->shader == MRT_SHADER_WHITTED || o->shader == MRT_SHADER_PATHTRACER || o->shader == MRT_SHADER_NOSHADOWS)) ||
        (job->camera.kind != MRT_CAMERA_PERSPECTIVE && job->camera.kind != MRT_CAMERA_ORTHOGRAPHIC) || o->pixel_sampler < 0 || o->pixel_sampler > 3 ||
        o->light_sampler < 0 || o->light_sampler > 3 || o->rr_sampler < 0 || o->rr_sampler > 3 || !job->bitmap) {
        set_error(ctx, "mrt_batch_submit: invalid options");
        return MRT_ERR_ARG;
    }
    if (!plain_rectangle(*o, job->stride_bytes)) {
        set_error(ctx, "mrt_batch_submit: width must be a multiple of 16 with stride_bytes = 4 * width and "
                       "height / (height / 16) == 16");
        return MRT_ERR_ARG;
    }
    if (!direct_shader(o->shader) && (o->depth_max > (int)b->opts.max_depth || o->spl > b->opts.max_spl)) {
        set_error(ctx, "mrt_batch_submit: depth_max above the batch's max_depth (%u) or samplesLight above max_spl (%u)",
                  b->opts.max_depth, b->opts.max_spl);
        return MRT_ERR_ARG;
    }
    if (((uintptr_t)job->bitmap & 3u) || ((uintptr_t)job->accum & 15u)) {
        set_error(ctx, "mrt_batch_submit: bitmap must be 4-byte aligned and the sums 16-byte aligned");
        return MRT_ERR_ARG;
    }
    const uint64_t n_tasks = (uint64_t)o->width * 16u * (o->height / 16u);
    const uint64_t total = n_tasks * o->spp;
    if (total > 0xFFFFFFFFull) { set_error(ctx, "mrt_batch_submit: more than 2^32 paths in one job"); return MRT_ERR_ARG; }
    const uint32_t slot = (uint32_t)(b->next_id % b->max_jobs);
    if (b->slots[slot].live) {
        int st = retire(b, false);
        if (st != MRT_OK) return st;
        if (b->slots[slot].live) { set_error(ctx, "mrt_batch_submit: %u jobs outstanding", b->max_jobs); return MRT_ERR_LIMIT; }
    }
    RenderParams p{};
    p.cam = make_camera(job->camera);
    p.width = o->width; p.height = o->height; p.spp = o->spp; p.spl = o->spl; p.stride_px = o->width;
    p.pixel_sampler = o->pixel_sampler; p.light_sampler = o->light_sampler; p.rr_sampler = o->rr_sampler;
    p.shader = o->shader; p.constant_value = o->constant_value;
    p.depth_min = o->depth_min; p.depth_max = o->depth_max;
    p.seed = o->seed; p.spp_offset = o->spp_offset;
    p.strata = o->spp;
    p.task_base = 0;
    p.tasks = nullptr;
    p.n_tasks = (uint32_t)n_tasks;
    p.bitmap = job->bitmap;
    p.accum = (float4 *)job->accum;
    p.inv_w = 1.0f / (float)o->width;   // Renderer.cpp:68-71
    p.inv_h = 1.0f / (float)o->height;
    p.pw = 0.5f / (float)o->width;
    p.ph = 0.5f / (float)o->height;
    p.depth_point = V3{o->depth_point[0], o->depth_point[1], o->depth_point[2]};
    b->h_jobs[slot] = p;
    b->h_scenes[slot] = s->dev;
    b->h_scenes[slot].error_flag = ctx->d_error;
    cudaStream_t q = ctx->stream;
    int st = cuda_status(ctx, cudaMemcpyAsync((RenderParams *)b->d_jobs.ptr + slot, &b->h_jobs[slot], sizeof(RenderParams),
                                              cudaMemcpyHostToDevice, q), "job upload");
    if (st == MRT_OK)
        st = cuda_status(ctx, cudaMemcpyAsync((DevScene *)b->d_scenes.ptr + slot, &b->h_scenes[slot], sizeof(DevScene),
                                              cudaMemcpyHostToDevice, q), "job upload");
    if (st == MRT_OK) st = cuda_status(ctx, cudaEventRecord(b->ev_jobs, q), "job upload");
    if (st != MRT_OK) return st;
    ++b->jobs_uploaded;
    MrtBatch::Job &j = b->slots[slot];
    j.id = b->next_id++;
    j.total = total;
    j.next = 0;
    j.live = true;
    b->active.push_back(slot);
    if (job_id) *job_id = j.id;
    return MRT_OK;
}

int mrt_batch_step(MrtBatch *b, uint32_t max_waves, uint32_t *launched) {
    if (!b) return MRT_ERR_ARG;
    if (launched) *launched = 0;
    MrtContext *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    int st = MRT_OK;
    if (!b->tuned && !b->active.empty()) {
        st = autotune(b);
        if (st == MRT_OK) st = check_batch_error(b);
        if (st != MRT_OK) return st;
        b->tuned = true;
    }
    for (uint32_t k = 0; k < max_waves && !b->active.empty(); ++k) {
        // bounded run-ahead: the ring slot is free once the wave kRing back has completed
        if (b->waves_launched - b->waves_done >= kRing) {
            st = retire(b, true);
            if (st != MRT_OK) return st;
        }
        const int64_t w = b->waves_launched;
        const int r = (int)(w % kRing);
        const int pipe = (int)(w % b->n_pipes);
        WaveDesc &d = b->h_desc[r];
        const uint32_t n = plan_wave(b, d, b->wave_roots, true, w, b->opts.policy);
        if (n == 0) break;
        if (b->waves_launched == b->waves_done) cudaEventRecord(b->ev_first, b->pipes[pipe].stream);
        uint32_t threads = b->block_threads, bps = b->blocks_per_sm;
        if (b->opts.kernel == 0 && b->n_levels <= kPathFrames && whole_paths_wave(d)) {
            threads = 0;
            bps = 8;
            ++b->waves_paths;
        }
        st = run_wave(b, d, pipe, threads, bps, r, w > b->waves_done ? (int)((w - 1) % kRing) : -1);
        if (st != MRT_OK) return st;
        b->paths += n;
        ++b->waves_launched;
        if (launched) ++*launched;
    }
    return retire(b, false);
}

int mrt_batch_completed(MrtBatch *b, uint64_t *ids, uint32_t capacity, uint32_t *count) {
    if (!b || !count || (capacity && !ids)) return MRT_ERR_ARG;
    int st = retire(b, false);
    if (st != MRT_OK) return st;
    const uint32_t n = (uint32_t)std::min<size_t>(capacity, b->newly_done.size());
    for (uint32_t i = 0; i < n; ++i) ids[i] = b->newly_done[i];
    b->newly_done.erase(b->newly_done.begin(), b->newly_done.begin() + n);
    *count = n;
    return MRT_OK;
}

int mrt_batch_run(MrtBatch *b) {
    if (!b) return MRT_ERR_ARG;
    int st = MRT_OK;
    while (st == MRT_OK && !b->active.empty()) {
        uint32_t n = 0;
        st = mrt_batch_step(b, kRing, &n);
    }
    while (st == MRT_OK && b->waves_done < b->waves_launched) st = retire(b, true);
    if (st == MRT_OK) st = check_batch_error(b);
    return st;
}

int mrt_batch_stats(const MrtBatch *b, MrtBatchStats *out) {
    if (!b || !out) return MRT_ERR_ARG;
    unsigned long long c[4] = {0, 0, 0, 0};
    cudaSetDevice(b->ctx->device);
    const int st = read_counters(const_cast<MrtBatch *>(b), c);
    if (st != MRT_OK) return st;
    out->rays_closest = c[0];
    out->rays_shadow = c[1];
    out->paths = b->paths;
    out->waves = (uint64_t)b->waves_launched;
    out->jobs_submitted = b->next_id;
    out->jobs_done = b->jobs_done;
    out->busy_ms = b->busy_ms;
    out->wave_roots = b->wave_roots;
    out->block_threads = b->block_threads;
    out->blocks_per_sm = b->blocks_per_sm;
    out->autotuned = b->autotuned;
    out->pipelines = b->n_pipes;
    out->kernel = b->block_threads == 0 ? MRT_BATCH_KERNEL_PATHS : MRT_BATCH_KERNEL_WAVEFRONT;
    out->waves_paths = b->block_threads == 0 ? (uint64_t)b->waves_launched : b->waves_paths;
    return MRT_OK;
}

}  // extern "C"
