// mrt_internal.h - host-side state behind the C ABI (not part of the public interface).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/mrt_cuda.h"
#include "mrt_device.cuh"

struct MrtArena;

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    MrtArena *arena = nullptr;   // carved from this arena (nullptr: cudaMalloc)
};

// One device allocation carved into the buffers of many scenes (geometry, trees, build scratch):
// best-fit blocks of 256-byte granularity with coalescing on free.  Thread-safe; no CUDA call after
// creation, so scene builds and evictions never synchronise the device.
struct MrtArena {
    int device = 0;
    char *base = nullptr;
    size_t capacity = 0;
    std::mutex mu;
    std::map<size_t, size_t> free_by_offset;          // offset -> size
    std::multimap<size_t, size_t> free_by_size;       // size -> offset
    size_t used = 0, peak = 0, live = 0;
};

struct MrtContext {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string error;
    int sm_count = 148;
    int32_t *d_error = nullptr;         // device error flag (MRT_ERR_LIMIT from kernels)
    uint32_t *d_counters = nullptr;     // work counters of the persistent kernels (64 slots)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    static constexpr int kTraceEvents = 16;             // start / end pairs around traversal launches
    cudaEvent_t trace_ev[2 * kTraceEvents] = {};
    cudaEvent_t wave_ev[2] = {nullptr, nullptr};   // the last two waves of a render (bounded run-ahead)
    static constexpr int kHostBands = 8;           // row bands a host-memory frame is shaded and copied out in
    cudaStream_t copy_stream = nullptr;            // device-to-host copies of finished bands
    cudaEvent_t band_ev[kHostBands] = {};
    // reusable scratch for host-pointer calls
    DevBuf scratch[4];
    MrtArena *arena = nullptr;          // device allocations of this context come from here when set
    // render scratch shared by the context's scenes (renders on one context are serialised on its
    // stream): wavefront queues, per-sample values, host-path bitmap staging
    DevBuf wave[8];
    // raster preview scratch: depth keys, queued large triangles, counters, host-path bitmap, overflow lists
    DevBuf raster[5];
};

struct RefBvhHost {
    std::vector<mrt::RefNode> nodes;
};

struct MrtScene {
    MrtContext *ctx = nullptr;
    mrt::DevScene dev{};
    // geometry
    uint32_t n_tri = 0, n_sph = 0, n_pln = 0, n_light = 0, n_mat = 0;
    DevBuf tri_a, tri_ab, tri_ac, tri_n, tri_c, tri_mat, sph, sph_mat, pln_n, pln_p, pln_mat, lights, mats;
    bool mixed_materials = false;       // some material reflects or transmits (per-material shade queues)
    // accelerators
    bool built = false;
    MrtAccelOpts opts{};
    DevBuf fnodes, ftris;
    uint64_t fnode_count = 0;
    DevBuf rnodes[3];
    uint64_t rnode_count[3] = {0, 0, 0};
    DevBuf grid_start[3], grid_refs[3], grid_trec;
    uint64_t grid_refs_count[3] = {0, 0, 0};
    // host copies needed by the reference-tree build and the grid bounds
    std::vector<float> h_abc;           // 9 floats per triangle
    std::vector<float> h_sph;           // 4 per sphere
    std::vector<float> h_pln;           // 6 per plane (point, normalised normal)
    // render state
    std::atomic<uint32_t> progress{0};
    std::atomic<int> stop{0};
    DevBuf work[1];                     // the scene's explicit pixel-task list (irregular image sizes)
    void *plan_cache = nullptr;         // pixel schedule of the last (width, height, pitch)
    void (*plan_cache_free)(void *) = nullptr;
    ~MrtScene() {
        if (plan_cache && plan_cache_free) plan_cache_free(plan_cache);
    }
};

namespace mrt_host {

bool set_error(MrtContext *ctx, const char *fmt, ...);
int cuda_status(MrtContext *ctx, cudaError_t e, const char *what);
int dev_alloc(MrtContext *ctx, DevBuf &b, size_t bytes);
void dev_free(DevBuf &b);
int ensure(MrtContext *ctx, DevBuf &b, size_t bytes);   // grow-only scratch
int check_kernel_error(MrtContext *ctx);                // reads and clears the device error flag

// builds (mrt_bvh.cu, mrt_grid.cu)
int build_fast_bvh(MrtScene *s);
int build_reference_bvh(MrtScene *s);
int build_grids(MrtScene *s, const float *camera_min, const float *camera_max, int grid_size, int grid_index);

// kernels (mrt_kernels.cu)
int launch_trace_closest(MrtScene *s, const MrtRay *d_rays, uint32_t n, MrtHit *d_hits);
int launch_trace_any(MrtScene *s, const MrtRay *d_rays, const float *d_dist, uint32_t n, uint8_t *d_occ);
int launch_trace_counts(MrtScene *s, const MrtRay *d_rays, uint32_t n, uint32_t *d_nodes, uint32_t *d_tris);
// Page-locked host buffers of an mrt_render call on the plain rectangle (row pitch 4 * width, the
// block schedule = the first n_tasks pixels): a render whose shading runs in whole 16-row stripes may
// shade them in bands and copy each band out on the context's copy stream while the next is shaded.
// `queued` is set once any copy is on that stream (the caller must then wait for it), `rows_done`
// once every scheduled pixel's copy is (the caller then copies nothing more).
struct HostOut {
    uint32_t *bitmap = nullptr;
    float *accum = nullptr;   // host sums or nullptr
    bool queued = false;
    bool rows_done = false;
};
int render(MrtScene *s, const MrtCamera *cam, const MrtRenderOpts *o, uint32_t *d_bitmap, uint32_t stride,
           float *d_accum, MrtRenderStats *stats, HostOut *out = nullptr);

mrt::DevCamera make_camera(const MrtCamera &c);
void camera_box(const MrtCamera &c, float *mn, float *mx);

}  // namespace mrt_host
