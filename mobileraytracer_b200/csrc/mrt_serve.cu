// mrt_serve.cu - the served form at the C ABI: render requests that arrive over time, on the batched
// renderer (continuous batching), for a host that cannot run the Python request loop.
//
// The reference renders one frame per Renderer::renderFrame call (Renderer.cpp:31-59) and, as a
// library, leaves the rest to its caller (the CLI's RayTrace(..., async, ...) hands one render to a
// detached thread, app/System_dependent/Linux/c_wrapper.cpp:535-548).  A service rendering many
// users' scenes needs what this file adds on top of mrt_batch_*:
//   * admission by device footprint: a request whose scene is not resident is admitted when the
//     scene's estimated footprint (geometry + tree, 240 bytes per triangle + 1 MiB, then the exact
//     size after the build) plus its image fits the budget; idle resident scenes are evicted, least
//     recently used first, to make room; a request that does not fit yet waits at the head of the
//     queue (arrival order);
//   * resident scenes and images: a scene stays on the device after its render together with its
//     image (the running mean), so a progressive re-render (spp_offset > 0) continues it without an
//     upload or a build; an evicted scene's image is kept on the host and restored with the scene;
//   * one render at a time per scene (requests of one scene run in arrival order), any number of
//     scenes at once: every dispatched request joins the batch's next waves beside the rays of the
//     requests already running.
// Scenes are built on a context that carves from the serve's arena and moved to the rendering
// context (mrt_scene_move), as the Python request loop does (serve.py); builds run in
// mrt_serve_poll, synchronously, while earlier waves keep the device busy.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <vector>

#include "mrt_internal.h"

using namespace mrt_host;

namespace {

using Clock = std::chrono::steady_clock;

struct ServeScene {
    // host copy of the caller's arrays
    std::vector<float> abc, nrm, col, sph, pln;
    std::vector<int32_t> tmat, smat, pmat;
    std::vector<MrtMaterial> mats;
    std::vector<MrtLightDesc> lights;
    MrtSceneDesc desc{};
    MrtAccelOpts accel{};
    MrtCamera accel_cam{};
    bool has_cam = false;
    // device state
    MrtScene *dev = nullptr;      // resident when set
    uint64_t bytes = 0;           // accounted bytes (scene + image)
    DevBuf image;                 // running mean of the scene's image
    uint32_t w = 0, h = 0;
    std::vector<uint32_t> saved;  // the image while the scene is evicted (a later re-render continues it)
    uint32_t saved_w = 0, saved_h = 0;
    bool busy = false;            // a request of this scene is in the batch
    std::deque<uint64_t> waiting; // admitted requests, arrival order
    std::list<uint64_t>::iterator lru_pos;
    bool in_lru = false;
};

struct ServeRequest {
    uint64_t scene = 0;
    MrtCamera cam{};
    MrtRenderOpts opts{};
    uint32_t *host_bitmap = nullptr;
    Clock::time_point arrival;
    double latency = -1.0;
};

template <class T>
void copy_array(std::vector<T> &dst, const T *src, size_t n) {
    if (src && n) dst.assign(src, src + n);
    else dst.clear();
}

uint64_t scene_estimate(const ServeScene &s) { return 240ull * s.desc.n_triangles + (1ull << 20); }

}  // namespace

struct MrtServe {
    MrtContext *render_ctx = nullptr;
    MrtContext *build_ctx = nullptr;
    MrtArena *arena = nullptr;
    MrtBatch *batch = nullptr;
    uint64_t budget = 0, used = 0, peak = 0;
    uint64_t next_scene = 1, next_req = 1;
    std::map<uint64_t, ServeScene> scenes;
    std::map<uint64_t, ServeRequest> reqs;
    std::deque<uint64_t> pending;             // submitted, not admitted
    std::list<uint64_t> idle;                 // resident scenes without work, least recently used first
    std::map<uint64_t, uint64_t> job_req;     // batch job -> request
    std::deque<uint64_t> finished;            // done, not reported yet
    MrtServeStats stats{};
};

namespace {

void lru_touch(MrtServe *sv, uint64_t sid, bool idle_now) {
    ServeScene &s = sv->scenes[sid];
    if (s.in_lru) { sv->idle.erase(s.lru_pos); s.in_lru = false; }
    if (idle_now && s.dev && !s.busy && s.waiting.empty()) {
        s.lru_pos = sv->idle.insert(sv->idle.end(), sid);
        s.in_lru = true;
    }
}

void release_scene(MrtServe *sv, ServeScene &s) {
    if (s.image.ptr && s.w && s.h) {   // keep the running mean on the host for a later re-render
        s.saved.resize((size_t)s.w * s.h);
        if (cudaMemcpy(s.saved.data(), s.image.ptr, 4ull * s.w * s.h, cudaMemcpyDeviceToHost) == cudaSuccess) {
            s.saved_w = s.w;
            s.saved_h = s.h;
        } else {
            s.saved.clear();
            s.saved_w = s.saved_h = 0;
        }
    }
    if (s.dev) mrt_scene_destroy(s.dev);
    s.dev = nullptr;
    dev_free(s.image);
    s.w = s.h = 0;
    sv->used -= std::min<uint64_t>(sv->used, s.bytes);
    s.bytes = 0;
}

bool evict_one(MrtServe *sv) {
    if (sv->idle.empty()) return false;
    const uint64_t sid = sv->idle.front();
    sv->idle.pop_front();
    ServeScene &s = sv->scenes[sid];
    s.in_lru = false;
    release_scene(sv, s);
    sv->stats.evictions++;
    return true;
}

// the scene of the request at the head of the queue made resident: 0 done, 1 wait (no room yet), <0 error
int make_resident(MrtServe *sv, ServeScene &s, const MrtRenderOpts &o) {
    const uint64_t image = 4ull * o.width * o.height;
    const uint64_t need = scene_estimate(s) + image;
    while (sv->used + need > sv->budget && evict_one(sv)) {
    }
    if (sv->used + need > sv->budget) return 1;
    int st = mrt_scene_create(sv->build_ctx, &s.desc, &s.dev);
    if (st == MRT_OK) {
        MrtAccelOpts a = s.accel;
        if (s.has_cam) a.camera = &s.accel_cam;
        st = mrt_scene_build(s.dev, &a);
    }
    if (st == MRT_OK) st = dev_alloc(sv->build_ctx, s.image, image);
    if (st == MRT_OK) st = mrt_scene_move(s.dev, sv->render_ctx);
    if (st != MRT_OK) {
        if (s.dev) mrt_scene_destroy(s.dev);
        s.dev = nullptr;
        dev_free(s.image);
        if (st == MRT_ERR_OOM) {
            // room may come back when other scenes finish or go idle; with nothing running and
            // nothing resident it never will
            if (evict_one(sv) || !sv->job_req.empty()) return 1;
            return sv->used == 0 ? -MRT_ERR_OOM : 1;
        }
        return -st;
    }
    s.w = o.width;
    s.h = o.height;
    if (!s.saved.empty() && s.saved_w == s.w && s.saved_h == s.h) {   // the image it had when evicted
        st = cuda_status(sv->render_ctx, cudaMemcpy(s.image.ptr, s.saved.data(), image, cudaMemcpyHostToDevice),
                         "serve image restore");
        if (st != MRT_OK) return -st;
    }
    s.saved.clear();
    s.saved_w = s.saved_h = 0;
    s.bytes = mrt_scene_device_bytes(s.dev) + image;
    sv->used += s.bytes;
    sv->peak = std::max(sv->peak, sv->used);
    sv->stats.builds++;
    return 0;
}

int dispatch(MrtServe *sv, uint64_t sid) {
    ServeScene &s = sv->scenes[sid];
    if (!s.dev || s.busy || s.waiting.empty()) return MRT_OK;
    const uint64_t rid = s.waiting.front();
    ServeRequest &r = sv->reqs[rid];
    const uint64_t bytes = 4ull * r.opts.width * r.opts.height;
    if (r.opts.width != s.w || r.opts.height != s.h) {   // a new image size: a new image
        dev_free(s.image);
        sv->used -= std::min<uint64_t>(sv->used, 4ull * s.w * s.h);
        int st = dev_alloc(sv->build_ctx, s.image, bytes);
        if (st != MRT_OK) return st;
        sv->used += bytes;
        s.bytes = s.bytes - 4ull * s.w * s.h + bytes;
        s.w = r.opts.width;
        s.h = r.opts.height;
    }
    if (r.opts.spp_offset == 0) {   // a first render starts from a cleared image (done before the batch's streams read it)
        int st = cuda_status(sv->render_ctx, cudaMemsetAsync(s.image.ptr, 0, bytes, sv->render_ctx->stream), "serve image");
        if (st == MRT_OK) st = cuda_status(sv->render_ctx, cudaStreamSynchronize(sv->render_ctx->stream), "serve image");
        if (st != MRT_OK) return st;
    }
    MrtBatchJob job{};
    job.scene = s.dev;
    job.camera = r.cam;
    job.opts = r.opts;
    job.bitmap = static_cast<uint32_t *>(s.image.ptr);
    job.stride_bytes = 4u * r.opts.width;
    job.accum = nullptr;
    uint64_t jid = 0;
    int st = mrt_batch_submit(sv->batch, &job, &jid);
    if (st != MRT_OK) return st;
    s.waiting.pop_front();
    s.busy = true;
    lru_touch(sv, sid, false);
    sv->job_req[jid] = rid;
    return MRT_OK;
}

}  // namespace

extern "C" {

int mrt_serve_create(int device, const MrtServeOpts *opts, MrtServe **out) {
    if (!opts || !out || opts->budget_bytes < (16ull << 20)) return MRT_ERR_ARG;
    auto *sv = new MrtServe();
    sv->budget = opts->budget_bytes;
    int st = mrt_context_create(device, &sv->render_ctx);
    if (st == MRT_OK) st = mrt_context_create(device, &sv->build_ctx);
    if (st == MRT_OK) st = mrt_arena_create(device, opts->budget_bytes + opts->build_slack_bytes, &sv->arena);
    if (st == MRT_OK) st = mrt_context_set_arena(sv->build_ctx, sv->arena);
    if (st == MRT_OK) st = mrt_batch_create(sv->render_ctx, &opts->batch, &sv->batch);
    if (st != MRT_OK) {
        mrt_serve_destroy(sv);
        return st;
    }
    *out = sv;
    return MRT_OK;
}

void mrt_serve_destroy(MrtServe *sv) {
    if (!sv) return;
    if (sv->batch) {
        mrt_batch_run(sv->batch);
        mrt_batch_destroy(sv->batch);
    }
    for (auto &kv : sv->scenes) {
        if (kv.second.dev) mrt_scene_destroy(kv.second.dev);
        dev_free(kv.second.image);
    }
    if (sv->build_ctx) mrt_context_destroy(sv->build_ctx);
    if (sv->render_ctx) mrt_context_destroy(sv->render_ctx);
    if (sv->arena) mrt_arena_destroy(sv->arena);
    delete sv;
}

const char *mrt_serve_error(const MrtServe *sv) {
    if (!sv) return "no serve";
    const char *a = mrt_context_error(sv->render_ctx);
    return (a && *a) ? a : mrt_context_error(sv->build_ctx);
}

int mrt_serve_add_scene(MrtServe *sv, const MrtSceneDesc *d, const MrtAccelOpts *accel, uint64_t *scene_id) {
    if (!sv || !d || !accel || !scene_id) return MRT_ERR_ARG;
    const uint64_t sid = sv->next_scene++;
    ServeScene &s = sv->scenes[sid];
    copy_array(s.abc, d->tri_abc, 9ull * d->n_triangles);
    copy_array(s.nrm, d->tri_normals, 9ull * d->n_triangles);
    copy_array(s.col, d->tri_colors, 9ull * d->n_triangles);
    copy_array(s.tmat, d->tri_material, (size_t)d->n_triangles);
    copy_array(s.sph, d->sphere_center_radius, 4ull * d->n_spheres);
    copy_array(s.smat, d->sphere_material, (size_t)d->n_spheres);
    copy_array(s.pln, d->plane_point_normal, 6ull * d->n_planes);
    copy_array(s.pmat, d->plane_material, (size_t)d->n_planes);
    copy_array(s.mats, d->materials, (size_t)d->n_materials);
    copy_array(s.lights, d->lights, (size_t)d->n_lights);
    s.desc = *d;
    s.desc.tri_abc = s.abc.empty() ? nullptr : s.abc.data();
    s.desc.tri_normals = s.nrm.empty() ? nullptr : s.nrm.data();
    s.desc.tri_colors = s.col.empty() ? nullptr : s.col.data();
    s.desc.tri_material = s.tmat.empty() ? nullptr : s.tmat.data();
    s.desc.sphere_center_radius = s.sph.empty() ? nullptr : s.sph.data();
    s.desc.sphere_material = s.smat.empty() ? nullptr : s.smat.data();
    s.desc.plane_point_normal = s.pln.empty() ? nullptr : s.pln.data();
    s.desc.plane_material = s.pmat.empty() ? nullptr : s.pmat.data();
    s.desc.materials = s.mats.empty() ? nullptr : s.mats.data();
    s.desc.lights = s.lights.empty() ? nullptr : s.lights.data();
    s.accel = *accel;
    if (accel->camera) { s.accel_cam = *accel->camera; s.has_cam = true; }
    s.accel.camera = nullptr;
    *scene_id = sid;
    return MRT_OK;
}

int mrt_serve_submit(MrtServe *sv, uint64_t scene_id, const MrtCamera *camera, const MrtRenderOpts *opts,
                     uint32_t *bitmap, uint64_t *request_id) {
    if (!sv || !camera || !opts || !bitmap || !request_id) return MRT_ERR_ARG;
    auto it = sv->scenes.find(scene_id);
    if (it == sv->scenes.end()) return MRT_ERR_ARG;
    if (opts->width < 16 || opts->height < 16 || opts->spp == 0 ||
        4ull * opts->width * opts->height + scene_estimate(it->second) > sv->budget)
        return MRT_ERR_ARG;   // never fits
    const uint64_t rid = sv->next_req++;
    ServeRequest &r = sv->reqs[rid];
    r.scene = scene_id;
    r.cam = *camera;
    r.opts = *opts;
    r.host_bitmap = bitmap;
    r.arrival = Clock::now();
    sv->pending.push_back(rid);
    sv->stats.submitted++;
    *request_id = rid;
    return MRT_OK;
}

int mrt_serve_poll(MrtServe *sv, uint64_t *done, uint32_t capacity, uint32_t *count) {
    if (!sv) return MRT_ERR_ARG;
    // 1. completed requests: the image to the caller's bitmap, the scene free for its next request
    std::vector<uint64_t> jobs(256);
    for (;;) {
        uint32_t n = 0;
        int st = mrt_batch_completed(sv->batch, jobs.data(), (uint32_t)jobs.size(), &n);
        if (st != MRT_OK) return st;
        for (uint32_t k = 0; k < n; ++k) {
            auto jr = sv->job_req.find(jobs[k]);
            if (jr == sv->job_req.end()) continue;
            const uint64_t rid = jr->second;
            sv->job_req.erase(jr);
            ServeRequest &r = sv->reqs[rid];
            ServeScene &s = sv->scenes[r.scene];
            st = cuda_status(sv->render_ctx, cudaMemcpyAsync(r.host_bitmap, s.image.ptr, 4ull * s.w * s.h,
                                                             cudaMemcpyDeviceToHost, sv->render_ctx->stream), "serve copy out");
            if (st == MRT_OK) st = cuda_status(sv->render_ctx, cudaStreamSynchronize(sv->render_ctx->stream), "serve copy out");
            if (st != MRT_OK) return st;
            r.latency = std::chrono::duration<double>(Clock::now() - r.arrival).count();
            s.busy = false;
            sv->finished.push_back(rid);
            sv->stats.completed++;
            lru_touch(sv, r.scene, true);
        }
        if (n < jobs.size()) break;
    }
    // 2. admission in arrival order
    while (!sv->pending.empty()) {
        const uint64_t rid = sv->pending.front();
        ServeRequest &r = sv->reqs[rid];
        ServeScene &s = sv->scenes[r.scene];
        if (!s.dev) {
            const int st = make_resident(sv, s, r.opts);
            if (st < 0) return -st;
            if (st > 0) break;    // no room yet: the head waits
        }
        s.waiting.push_back(rid);
        lru_touch(sv, r.scene, false);
        sv->pending.pop_front();
    }
    // 3. every resident scene with a request waiting and none running joins the batch
    for (auto &kv : sv->scenes) {
        int st = dispatch(sv, kv.first);
        if (st != MRT_OK) return st;
    }
    // 4. the next waves
    uint32_t launched = 0;
    int st = mrt_batch_step(sv->batch, 2, &launched);
    if (st != MRT_OK) return st;
    uint32_t n = 0;
    while (n < capacity && !sv->finished.empty()) {
        if (done) done[n] = sv->finished.front();
        sv->finished.pop_front();
        ++n;
    }
    if (count) *count = n;
    return MRT_OK;
}

int mrt_serve_pending(const MrtServe *sv, uint64_t *requests) {
    if (!sv || !requests) return MRT_ERR_ARG;
    uint64_t n = sv->pending.size() + sv->job_req.size() + sv->finished.size();
    for (const auto &kv : sv->scenes) n += kv.second.waiting.size();
    *requests = n;
    return MRT_OK;
}

int mrt_serve_request_latency(const MrtServe *sv, uint64_t request_id, double *seconds) {
    if (!sv || !seconds) return MRT_ERR_ARG;
    auto it = sv->reqs.find(request_id);
    if (it == sv->reqs.end() || it->second.latency < 0) return MRT_ERR_STATE;
    *seconds = it->second.latency;
    return MRT_OK;
}

int mrt_serve_stats(const MrtServe *sv, MrtServeStats *out) {
    if (!sv || !out) return MRT_ERR_ARG;
    *out = sv->stats;
    out->resident_bytes = sv->used;
    out->peak_bytes = sv->peak;
    MrtBatchStats b{};
    mrt_batch_stats(sv->batch, &b);
    out->rays_closest = b.rays_closest;
    out->rays_shadow = b.rays_shadow;
    return MRT_OK;
}

}  // extern "C"
