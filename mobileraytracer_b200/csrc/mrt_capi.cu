// mrt_capi.cu - the extern "C" entry points of include/mrt_cuda.h: context, scene upload,
// accelerator build dispatch and the trace entry points.  Rendering lives in mrt_render.cu.
#include <cstdarg>
#include <cstring>
#include <new>

#include "mrt_internal.h"

using namespace mrt;

namespace mrt_host {

bool set_error(MrtContext *ctx, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->error = buf;
    return false;
}

int cuda_status(MrtContext *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MRT_OK;
    set_error(ctx, "%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? MRT_ERR_OOM : MRT_ERR_CUDA;
}

static void arena_insert_free(MrtArena *a, size_t off, size_t size) {
    // coalesce with the free neighbours
    auto next = a->free_by_offset.lower_bound(off);
    if (next != a->free_by_offset.end() && off + size == next->first) {
        auto range = a->free_by_size.equal_range(next->second);
        for (auto it = range.first; it != range.second; ++it)
            if (it->second == next->first) { a->free_by_size.erase(it); break; }
        size += next->second;
        next = a->free_by_offset.erase(next);
    }
    if (next != a->free_by_offset.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            auto range = a->free_by_size.equal_range(prev->second);
            for (auto it = range.first; it != range.second; ++it)
                if (it->second == prev->first) { a->free_by_size.erase(it); break; }
            off = prev->first;
            size += prev->second;
            a->free_by_offset.erase(prev);
        }
    }
    a->free_by_offset[off] = size;
    a->free_by_size.emplace(size, off);
}

static void *arena_alloc(MrtArena *a, size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    std::lock_guard<std::mutex> lock(a->mu);
    auto it = a->free_by_size.lower_bound(bytes);   // best fit
    if (it == a->free_by_size.end()) return nullptr;
    const size_t size = it->first, off = it->second;
    a->free_by_size.erase(it);
    a->free_by_offset.erase(off);
    if (size > bytes) {
        a->free_by_offset[off + bytes] = size - bytes;
        a->free_by_size.emplace(size - bytes, off + bytes);
    }
    a->used += bytes;
    a->peak = std::max(a->peak, a->used);
    ++a->live;
    return a->base + off;
}

static void arena_free(MrtArena *a, void *p, size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    std::lock_guard<std::mutex> lock(a->mu);
    arena_insert_free(a, (size_t)((char *)p - a->base), bytes);
    a->used -= bytes;
    --a->live;
}

int dev_alloc(MrtContext *ctx, DevBuf &b, size_t bytes) {
    dev_free(b);
    if (bytes == 0) bytes = 16;
    if (ctx->arena) {
        b.ptr = arena_alloc(ctx->arena, bytes);
        if (!b.ptr) {
            size_t largest = 0;
            {
                std::lock_guard<std::mutex> lock(ctx->arena->mu);
                if (!ctx->arena->free_by_size.empty()) largest = ctx->arena->free_by_size.rbegin()->first;
            }
            set_error(ctx, "device arena: no free block of %zu bytes (used %zu of %zu, largest free block %zu)", bytes,
                      ctx->arena->used, ctx->arena->capacity, largest);
            return MRT_ERR_OOM;
        }
        b.bytes = bytes;
        b.arena = ctx->arena;
        return MRT_OK;
    }
    const cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) {
        b.ptr = nullptr;
        cudaGetLastError();
        set_error(ctx, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
        return MRT_ERR_OOM;
    }
    b.bytes = bytes;
    return MRT_OK;
}

void dev_free(DevBuf &b) {
    if (b.ptr) {
        if (b.arena) arena_free(b.arena, b.ptr, b.bytes);
        else cudaFree(b.ptr);
    }
    b.ptr = nullptr;
    b.bytes = 0;
    b.arena = nullptr;
}

int ensure(MrtContext *ctx, DevBuf &b, size_t bytes) {
    if (b.ptr && b.bytes >= bytes) return MRT_OK;
    return dev_alloc(ctx, b, bytes + bytes / 4);
}

int check_kernel_error(MrtContext *ctx) {
    int32_t flag = 0;
    cudaError_t e = cudaMemcpyAsync(&flag, ctx->d_error, sizeof(flag), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_status(ctx, e, "kernel");
    if (flag != 0) {
        cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), ctx->stream);
        set_error(ctx, "a traversal cap was exceeded (stack or step limit)");
        return flag;
    }
    return MRT_OK;
}

static V3 h_normalize(V3 v) { return normalize(v); }

DevCamera make_camera(const MrtCamera &c) {
    // Camera.cpp:52-57 and Perspective.cpp:10-15 (degToRad = deg * pi / 180, Camera.cpp:68-71)
    DevCamera k;
    k.position = V3{c.position[0], c.position[1], c.position[2]};
    k.direction = h_normalize(V3{c.look_at[0], c.look_at[1], c.look_at[2]} - k.position);
    k.right = cross(V3{c.up[0], c.up[1], c.up[2]}, k.direction);
    k.up = cross(k.direction, k.right);
    k.kind = c.kind;
    if (c.kind == MRT_CAMERA_ORTHOGRAPHIC) {   // Orthographic.cpp:12-17: half the film size
        k.hfov = c.fov_h_deg / 2.0f;
        k.vfov = c.fov_v_deg / 2.0f;
        return k;
    }
    const float pi = 3.14159265358979323846f;
    k.hfov = (c.fov_h_deg * pi) / 180.0f;
    k.vfov = (c.fov_v_deg * pi) / 180.0f;
    return k;
}

// Camera::getAABB (Camera.cpp:39-44: the position) and Orthographic::getAABB (Orthographic.cpp:36-46:
// two corners of the film rectangle, in the reference's order of operations)
void camera_box(const MrtCamera &c, float *mn, float *mx) {
    const DevCamera k = make_camera(c);
    V3 a = k.position, b = k.position;
    if (c.kind == MRT_CAMERA_ORTHOGRAPHIC) {
        a = (((k.position + (k.right * (0.0f - 0.5f)) * k.hfov) + k.right * -0.5f) + (k.up * (0.5f - 0.0f)) * k.vfov) +
            k.up * -0.5f;
        b = (((k.position + (k.right * (1.0f - 0.5f)) * k.hfov) + k.right * 0.5f) + (k.up * (0.5f - 1.0f)) * k.vfov) +
            k.up * 0.5f;
    }
    mn[0] = a.x; mn[1] = a.y; mn[2] = a.z;
    mx[0] = b.x; mx[1] = b.y; mx[2] = b.z;
}

}  // namespace mrt_host

using namespace mrt_host;

// ---------------------------------------------------------------------------------------------
// triangle preparation: Triangle constructors (Triangle.cpp:10-54) on the device
// ---------------------------------------------------------------------------------------------
__global__ void k_prepare_triangles(uint32_t n, const float *__restrict__ abc, const float *__restrict__ nin,
                                    const float *__restrict__ cin, const int32_t *__restrict__ min_,
                                    float4 *a4, float4 *ab4, float4 *ac4, float *nout, float *cout, int32_t *mout) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *p = abc + 9 * (size_t)i;
    const V3 A{p[0], p[1], p[2]}, B{p[3], p[4], p[5]}, C{p[6], p[7], p[8]};
    const V3 ac = C - A, ab = B - A;
    a4[i] = make_float4(A.x, A.y, A.z, 0.0f);
    ab4[i] = make_float4(ab.x, ab.y, ab.z, 0.0f);
    ac4[i] = make_float4(ac.x, ac.y, ac.z, 0.0f);
    float *no = nout + 9 * (size_t)i;
    if (nin) {
        for (int k = 0; k < 9; ++k) no[k] = nin[9 * (size_t)i + k];
    } else {
        const V3 nn = normalize(cross(ac, ab));
        for (int k = 0; k < 3; ++k) { no[3 * k] = nn.x; no[3 * k + 1] = nn.y; no[3 * k + 2] = nn.z; }
    }
    float *co = cout + 9 * (size_t)i;
    for (int k = 0; k < 9; ++k) co[k] = cin ? cin[9 * (size_t)i + k] : 0.0f;
    mout[i] = min_ ? min_[i] : -1;
}

extern "C" {

int mrt_context_create(int device, MrtContext **out) {
    if (!out) return MRT_ERR_ARG;
    *out = nullptr;
    MrtContext *ctx = new (std::nothrow) MrtContext();
    if (!ctx) return MRT_ERR_OOM;
    ctx->device = device;
    int st = cuda_status(ctx, cudaSetDevice(device), "cudaSetDevice");
    if (st == MRT_OK) st = cuda_status(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
    if (st == MRT_OK) st = cuda_status(ctx, cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device), "attr");
    if (st == MRT_OK) st = cuda_status(ctx, cudaMalloc(&ctx->d_error, sizeof(int32_t)), "cudaMalloc");
    if (st == MRT_OK) st = cuda_status(ctx, cudaMemset(ctx->d_error, 0, sizeof(int32_t)), "memset");
    if (st == MRT_OK) st = cuda_status(ctx, cudaMalloc(&ctx->d_counters, 64 * sizeof(uint32_t)), "cudaMalloc");
    if (st == MRT_OK) st = cuda_status(ctx, cudaEventCreate(&ctx->ev0), "event");
    if (st == MRT_OK) st = cuda_status(ctx, cudaEventCreate(&ctx->ev1), "event");
    for (auto &e : ctx->trace_ev)
        if (st == MRT_OK) st = cuda_status(ctx, cudaEventCreate(&e), "event");
    for (int k = 0; k < 2 && st == MRT_OK; ++k)
        st = cuda_status(ctx, cudaEventCreateWithFlags(&ctx->wave_ev[k], cudaEventDisableTiming), "event");
    for (auto &e : ctx->band_ev)
        if (st == MRT_OK) st = cuda_status(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    if (st == MRT_OK) st = cuda_status(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "stream");

    if (st != MRT_OK) {
        fprintf(stderr, "mrt_context_create: %s\n", ctx->error.c_str());
        mrt_context_destroy(ctx);
        return st;
    }
    *out = ctx;
    return MRT_OK;
}

void mrt_context_destroy(MrtContext *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    for (auto &b : ctx->scratch) dev_free(b);
    for (auto &b : ctx->wave) dev_free(b);
    for (auto &b : ctx->raster) dev_free(b);
    if (ctx->d_error) cudaFree(ctx->d_error);
    if (ctx->d_counters) cudaFree(ctx->d_counters);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (auto &e : ctx->trace_ev) if (e) cudaEventDestroy(e);
    for (auto &e : ctx->wave_ev) if (e) cudaEventDestroy(e);
    for (auto &e : ctx->band_ev) if (e) cudaEventDestroy(e);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *mrt_context_error(const MrtContext *ctx) { return ctx ? ctx->error.c_str() : "null context"; }

int mrt_arena_create(int device, uint64_t bytes, MrtArena **out) {
    if (!out || bytes == 0) return MRT_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return MRT_ERR_CUDA;
    MrtArena *a = new (std::nothrow) MrtArena();
    if (!a) return MRT_ERR_OOM;
    a->device = device;
    a->capacity = (size_t)(bytes & ~(uint64_t)255);
    if (cudaMalloc(&a->base, a->capacity) != cudaSuccess) {
        cudaGetLastError();
        delete a;
        return MRT_ERR_OOM;
    }
    a->free_by_offset[0] = a->capacity;
    a->free_by_size.emplace(a->capacity, 0);
    *out = a;
    return MRT_OK;
}

int mrt_arena_destroy(MrtArena *a) {
    if (!a) return MRT_OK;
    {
        std::lock_guard<std::mutex> lock(a->mu);
        if (a->live) return MRT_ERR_STATE;   // buffers still carved from it
    }
    cudaSetDevice(a->device);
    cudaFree(a->base);
    delete a;
    return MRT_OK;
}

int mrt_arena_stats(MrtArena *a, uint64_t *capacity, uint64_t *used, uint64_t *peak, uint64_t *largest_free) {
    if (!a) return MRT_ERR_ARG;
    std::lock_guard<std::mutex> lock(a->mu);
    if (capacity) *capacity = a->capacity;
    if (used) *used = a->used;
    if (peak) *peak = a->peak;
    if (largest_free) *largest_free = a->free_by_size.empty() ? 0 : a->free_by_size.rbegin()->first;
    return MRT_OK;
}

int mrt_context_set_arena(MrtContext *ctx, MrtArena *arena) {
    if (!ctx) return MRT_ERR_ARG;
    if (arena && arena->device != ctx->device) {
        set_error(ctx, "mrt_context_set_arena: arena on device %d, context on device %d", arena->device, ctx->device);
        return MRT_ERR_ARG;
    }
    ctx->arena = arena;
    return MRT_OK;
}

int mrt_context_synchronize(MrtContext *ctx) {
    if (!ctx) return MRT_ERR_ARG;
    return cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
}

void *mrt_context_stream(MrtContext *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

static void scene_free(MrtScene *s) {
    DevBuf *bufs[] = {&s->tri_a, &s->tri_ab, &s->tri_ac, &s->tri_n, &s->tri_c, &s->tri_mat, &s->sph, &s->sph_mat,
                      &s->pln_n, &s->pln_p, &s->pln_mat, &s->lights, &s->mats, &s->fnodes, &s->ftris};
    for (DevBuf *b : bufs) dev_free(*b);
    for (int k = 0; k < 3; ++k) { dev_free(s->rnodes[k]); dev_free(s->grid_start[k]); dev_free(s->grid_refs[k]); }
    dev_free(s->grid_trec);
    for (auto &b : s->work) dev_free(b);
}

int mrt_scene_create(MrtContext *ctx, const MrtSceneDesc *d, MrtScene **out) {
    if (!ctx || !d || !out) return MRT_ERR_ARG;
    *out = nullptr;
    if ((d->n_triangles && !d->tri_abc) || (d->n_spheres && !d->sphere_center_radius) ||
        (d->n_planes && !d->plane_point_normal) || (d->n_materials && !d->materials) || (d->n_lights && !d->lights)) {
        set_error(ctx, "mrt_scene_create: a non-empty array has a null pointer");
        return MRT_ERR_ARG;
    }
    if (d->n_triangles > 0x3FFFFFFFu || d->n_spheres > 0x3FFFFFFFu || d->n_planes > 0x3FFFFFFFu) {
        set_error(ctx, "mrt_scene_create: more than 2^30 primitives of one type");
        return MRT_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    MrtScene *s = new (std::nothrow) MrtScene();
    if (!s) return MRT_ERR_OOM;
    s->ctx = ctx;
    s->n_tri = d->n_triangles;
    s->n_sph = d->n_spheres;
    s->n_pln = d->n_planes;
    s->n_light = d->n_lights;
    s->n_mat = d->n_materials;
    for (uint32_t k = 0; k < d->n_materials; ++k) {
        const MrtMaterial &m = d->materials[k];
        if (m.ks[0] > 0 || m.ks[1] > 0 || m.ks[2] > 0 || m.kt[0] > 0 || m.kt[1] > 0 || m.kt[2] > 0) s->mixed_materials = true;
    }
    const uint32_t nt = s->n_tri;
    int st = MRT_OK;
    auto alloc = [&](DevBuf &b, size_t bytes) { if (st == MRT_OK) st = dev_alloc(ctx, b, bytes); };
    alloc(s->tri_a, 16ull * nt);
    alloc(s->tri_ab, 16ull * nt);
    alloc(s->tri_ac, 16ull * nt);
    alloc(s->tri_n, 36ull * nt);
    alloc(s->tri_c, 36ull * nt);
    alloc(s->tri_mat, 4ull * nt);
    alloc(s->sph, 16ull * s->n_sph);
    alloc(s->sph_mat, 4ull * s->n_sph);
    alloc(s->pln_n, 16ull * s->n_pln);
    alloc(s->pln_p, 16ull * s->n_pln);
    alloc(s->pln_mat, 4ull * s->n_pln);
    alloc(s->lights, sizeof(DevLight) * s->n_light);
    alloc(s->mats, sizeof(DevMaterial) * s->n_mat);
    // staging copies of the triangle inputs, then the constructor kernel
    DevBuf st_abc, st_n, st_c, st_m;
    alloc(st_abc, 36ull * nt);
    if (d->tri_normals) alloc(st_n, 36ull * nt);
    if (d->tri_colors) alloc(st_c, 36ull * nt);
    if (d->tri_material) alloc(st_m, 4ull * nt);
    cudaStream_t q = ctx->stream;
    if (st == MRT_OK && nt) {
        st = cuda_status(ctx, cudaMemcpyAsync(st_abc.ptr, d->tri_abc, 36ull * nt, cudaMemcpyHostToDevice, q), "upload");
        if (st == MRT_OK && d->tri_normals) st = cuda_status(ctx, cudaMemcpyAsync(st_n.ptr, d->tri_normals, 36ull * nt, cudaMemcpyHostToDevice, q), "upload");
        if (st == MRT_OK && d->tri_colors) st = cuda_status(ctx, cudaMemcpyAsync(st_c.ptr, d->tri_colors, 36ull * nt, cudaMemcpyHostToDevice, q), "upload");
        if (st == MRT_OK && d->tri_material) st = cuda_status(ctx, cudaMemcpyAsync(st_m.ptr, d->tri_material, 4ull * nt, cudaMemcpyHostToDevice, q), "upload");
        if (st == MRT_OK) {
            k_prepare_triangles<<<(nt + 255) / 256, 256, 0, q>>>(
                nt, (const float *)st_abc.ptr, d->tri_normals ? (const float *)st_n.ptr : nullptr,
                d->tri_colors ? (const float *)st_c.ptr : nullptr, d->tri_material ? (const int32_t *)st_m.ptr : nullptr,
                (float4 *)s->tri_a.ptr, (float4 *)s->tri_ab.ptr, (float4 *)s->tri_ac.ptr, (float *)s->tri_n.ptr,
                (float *)s->tri_c.ptr, (int32_t *)s->tri_mat.ptr);
            st = cuda_status(ctx, cudaGetLastError(), "k_prepare_triangles");
        }
    }
    // spheres (Sphere.cpp:13-16: sq_radius = radius * radius), planes (Plane.cpp:11-15)
    std::vector<float4> hs(s->n_sph), hpn(s->n_pln), hpp(s->n_pln);
    s->h_sph.resize(4ull * s->n_sph);
    for (uint32_t i = 0; i < s->n_sph; ++i) {
        const float *c = d->sphere_center_radius + 4 * i;
        hs[i] = make_float4(c[0], c[1], c[2], c[3] * c[3]);
        for (int k = 0; k < 4; ++k) s->h_sph[4 * i + k] = k < 3 ? c[k] : c[3] * c[3];
    }
    s->h_pln.resize(6ull * s->n_pln);
    for (uint32_t i = 0; i < s->n_pln; ++i) {
        const float *p = d->plane_point_normal + 6 * i;
        const V3 n = normalize(V3{p[3], p[4], p[5]});
        hpn[i] = make_float4(n.x, n.y, n.z, 0.0f);
        hpp[i] = make_float4(p[0], p[1], p[2], 0.0f);
        const float vals[6] = {p[0], p[1], p[2], n.x, n.y, n.z};
        for (int k = 0; k < 6; ++k) s->h_pln[6 * i + k] = vals[k];
    }
    std::vector<int32_t> sm(s->n_sph), pm(s->n_pln);
    for (uint32_t i = 0; i < s->n_sph; ++i) sm[i] = d->sphere_material ? d->sphere_material[i] : -1;
    for (uint32_t i = 0; i < s->n_pln; ++i) pm[i] = d->plane_material ? d->plane_material[i] : -1;
    std::vector<DevLight> hl(s->n_light);
    for (uint32_t i = 0; i < s->n_light; ++i) {
        const MrtLightDesc &l = d->lights[i];
        DevLight &o = hl[i];
        o.kind = l.kind;
        o.pos = V3{l.p0[0], l.p0[1], l.p0[2]};
        const V3 A{l.p0[0], l.p0[1], l.p0[2]}, B{l.p1[0], l.p1[1], l.p1[2]}, C{l.p2[0], l.p2[1], l.p2[2]};
        o.a = A;
        o.ab = B - A;
        o.ac = C - A;
        o.na = normalize(cross(o.ac, o.ab));
        const MrtMaterial &m = l.radiance;
        o.radiance = DevMaterial{V3{m.le[0], m.le[1], m.le[2]}, V3{m.kd[0], m.kd[1], m.kd[2]},
                                 V3{m.ks[0], m.ks[1], m.ks[2]}, V3{m.kt[0], m.kt[1], m.kt[2]}, m.ior};
        if (l.kind != MRT_LIGHT_POINT && l.kind != MRT_LIGHT_AREA) st = MRT_ERR_ARG;
    }
    std::vector<DevMaterial> hm(s->n_mat);
    for (uint32_t i = 0; i < s->n_mat; ++i) {
        const MrtMaterial &m = d->materials[i];
        hm[i] = DevMaterial{V3{m.le[0], m.le[1], m.le[2]}, V3{m.kd[0], m.kd[1], m.kd[2]},
                            V3{m.ks[0], m.ks[1], m.ks[2]}, V3{m.kt[0], m.kt[1], m.kt[2]}, m.ior};
    }
    auto up = [&](DevBuf &b, const void *src, size_t bytes) {
        if (st == MRT_OK && bytes) st = cuda_status(ctx, cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice, q), "upload");
    };
    up(s->sph, hs.data(), 16ull * s->n_sph);
    up(s->sph_mat, sm.data(), 4ull * s->n_sph);
    up(s->pln_n, hpn.data(), 16ull * s->n_pln);
    up(s->pln_p, hpp.data(), 16ull * s->n_pln);
    up(s->pln_mat, pm.data(), 4ull * s->n_pln);
    up(s->lights, hl.data(), sizeof(DevLight) * s->n_light);
    up(s->mats, hm.data(), sizeof(DevMaterial) * s->n_mat);
    if (st == MRT_OK) st = cuda_status(ctx, cudaStreamSynchronize(q), "scene upload");
    s->h_abc.assign(d->tri_abc, d->tri_abc + 9ull * nt);
    dev_free(st_abc); dev_free(st_n); dev_free(st_c); dev_free(st_m);
    if (st != MRT_OK) {
        if (ctx->error.empty()) set_error(ctx, "mrt_scene_create: invalid light kind");
        scene_free(s);
        delete s;
        return st;
    }
    DevScene &v = s->dev;
    v.n_tri = nt; v.n_sph = s->n_sph; v.n_pln = s->n_pln; v.n_light = s->n_light; v.n_mat = s->n_mat;
    v.tri_a = (const float4 *)s->tri_a.ptr; v.tri_ab = (const float4 *)s->tri_ab.ptr; v.tri_ac = (const float4 *)s->tri_ac.ptr;
    v.tri_n = (const float *)s->tri_n.ptr; v.tri_c = (const float *)s->tri_c.ptr; v.tri_mat = (const int32_t *)s->tri_mat.ptr;
    v.sph = (const float4 *)s->sph.ptr; v.sph_mat = (const int32_t *)s->sph_mat.ptr;
    v.pln_n = (const float4 *)s->pln_n.ptr; v.pln_p = (const float4 *)s->pln_p.ptr; v.pln_mat = (const int32_t *)s->pln_mat.ptr;
    v.lights = (const DevLight *)s->lights.ptr; v.mats = (const DevMaterial *)s->mats.ptr;
    v.error_flag = ctx->d_error;
    *out = s;
    return MRT_OK;
}

void mrt_scene_destroy(MrtScene *s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    scene_free(s);
    delete s;
}

int mrt_scene_move(MrtScene *s, MrtContext *ctx) {
    if (!s || !ctx) return MRT_ERR_ARG;
    if (ctx->device != s->ctx->device) {
        set_error(ctx, "mrt_scene_move: scene on device %d, context on device %d", s->ctx->device, ctx->device);
        return MRT_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    const int st = cuda_status(ctx, cudaStreamSynchronize(s->ctx->stream), "mrt_scene_move");
    if (st != MRT_OK) return st;
    s->ctx = ctx;
    s->dev.error_flag = ctx->d_error;
    return MRT_OK;
}

int mrt_scene_build(MrtScene *s, const MrtAccelOpts *o) {
    if (!s || !o) return MRT_ERR_ARG;
    MrtContext *ctx = s->ctx;
    cudaSetDevice(ctx->device);
    if (o->accelerator < MRT_ACCEL_NAIVE || o->accelerator > MRT_ACCEL_BVH || o->bvh_mode < 0 || o->bvh_mode > 1 ||
        o->grid_index < 0 || o->grid_index > 1 || o->grid_size < 0 || o->grid_size > 1024) {
        set_error(ctx, "mrt_scene_build: invalid options");
        return MRT_ERR_ARG;
    }
    s->built = false;
    s->opts = *o;
    dev_free(s->fnodes);
    dev_free(s->ftris);
    for (int k = 0; k < 3; ++k) { dev_free(s->rnodes[k]); dev_free(s->grid_start[k]); dev_free(s->grid_refs[k]); }
    dev_free(s->grid_trec);
    s->dev.grid[kTriangle].trec = nullptr;
    s->dev.accel = o->accelerator;
    s->dev.bvh_mode = o->bvh_mode;
    int st = MRT_OK;
    if (o->accelerator == MRT_ACCEL_BVH) st = o->bvh_mode == MRT_BVH_FAST ? build_fast_bvh(s) : build_reference_bvh(s);
    else if (o->accelerator == MRT_ACCEL_REGULAR_GRID) {
        float cmn[3] = {o->camera_position[0], o->camera_position[1], o->camera_position[2]};
        float cmx[3] = {cmn[0], cmn[1], cmn[2]};
        if (o->camera) camera_box(*o->camera, cmn, cmx);
        st = build_grids(s, cmn, cmx, o->grid_size, o->grid_index);
    }
    if (st != MRT_OK) return st;
    st = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "mrt_scene_build");
    if (st == MRT_OK) s->built = true;
    return st;
}

uint64_t mrt_scene_device_bytes(const MrtScene *s) {
    if (!s) return 0;
    uint64_t t = 0;
    const DevBuf *bufs[] = {&s->tri_a, &s->tri_ab, &s->tri_ac, &s->tri_n, &s->tri_c, &s->tri_mat, &s->sph, &s->sph_mat,
                            &s->pln_n, &s->pln_p, &s->pln_mat, &s->lights, &s->mats, &s->fnodes, &s->ftris};
    for (const DevBuf *b : bufs) t += b->bytes;
    for (int k = 0; k < 3; ++k) t += s->rnodes[k].bytes + s->grid_start[k].bytes + s->grid_refs[k].bytes;
    t += s->grid_trec.bytes;
    return t;
}

int mrt_scene_accel_info(const MrtScene *s, uint64_t *nodes, uint64_t *refs, int32_t *grid_size) {
    if (!s) return MRT_ERR_ARG;
    if (nodes) *nodes = s->opts.accelerator == MRT_ACCEL_BVH
                            ? (s->opts.bvh_mode == MRT_BVH_FAST ? s->fnode_count : s->rnode_count[kTriangle])
                            : (uint64_t)s->dev.grid[kTriangle].G * s->dev.grid[kTriangle].G * s->dev.grid[kTriangle].G;
    if (refs) *refs = s->grid_refs_count[kTriangle];
    if (grid_size) *grid_size = s->dev.grid[kTriangle].G;
    return MRT_OK;
}

// host/device pointer plumbing for the trace entry points
static int stage_in(MrtContext *ctx, DevBuf &b, const void *src, size_t bytes) {
    int st = ensure(ctx, b, bytes);
    if (st != MRT_OK) return st;
    return cuda_status(ctx, cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice, ctx->stream), "copy in");
}

// device buffers are read and written with vector accesses: rays as two 16-byte loads, hits as
// one 8-byte store, per-ray counters and distances as 4-byte words
static bool misaligned(MrtContext *ctx, uint32_t mem, const void *p, uintptr_t align, const char *what) {
    if (mem != MRT_MEM_DEVICE || ((uintptr_t)p & (align - 1)) == 0) return false;
    set_error(ctx, "%s must be %u-byte aligned", what, (unsigned)align);
    return true;
}

int mrt_trace_closest(MrtScene *s, const MrtRay *rays, uint32_t n, MrtHit *hits, uint32_t mem) {
    if (!s || (n && (!rays || !hits))) return MRT_ERR_ARG;
    MrtContext *ctx = s->ctx;
    if (misaligned(ctx, mem, rays, 16, "rays") || misaligned(ctx, mem, hits, 8, "hits")) return MRT_ERR_ARG;
    if (!s->built) { set_error(ctx, "mrt_trace_closest before mrt_scene_build"); return MRT_ERR_STATE; }
    if (n == 0) return MRT_OK;
    cudaSetDevice(ctx->device);
    const MrtRay *d_rays = rays;
    MrtHit *d_hits = hits;
    int st = MRT_OK;
    if (mem == MRT_MEM_HOST) {
        st = stage_in(ctx, ctx->scratch[0], rays, sizeof(MrtRay) * (size_t)n);
        if (st == MRT_OK) st = ensure(ctx, ctx->scratch[1], sizeof(MrtHit) * (size_t)n);
        if (st != MRT_OK) return st;
        d_rays = (const MrtRay *)ctx->scratch[0].ptr;
        d_hits = (MrtHit *)ctx->scratch[1].ptr;
    }
    st = launch_trace_closest(s, d_rays, n, d_hits);
    if (st == MRT_OK && mem == MRT_MEM_HOST)
        st = cuda_status(ctx, cudaMemcpyAsync(hits, d_hits, sizeof(MrtHit) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
    if (st == MRT_OK) st = check_kernel_error(ctx);
    return st;
}

int mrt_trace_any(MrtScene *s, const MrtRay *rays, const float *dist, uint32_t n, uint8_t *occluded, uint32_t mem) {
    if (!s || (n && (!rays || !dist || !occluded))) return MRT_ERR_ARG;
    MrtContext *ctx = s->ctx;
    if (misaligned(ctx, mem, rays, 16, "rays") || misaligned(ctx, mem, dist, 4, "dist")) return MRT_ERR_ARG;
    if (!s->built) { set_error(ctx, "mrt_trace_any before mrt_scene_build"); return MRT_ERR_STATE; }
    if (n == 0) return MRT_OK;
    cudaSetDevice(ctx->device);
    const MrtRay *d_rays = rays;
    const float *d_dist = dist;
    uint8_t *d_occ = occluded;
    int st = MRT_OK;
    if (mem == MRT_MEM_HOST) {
        st = stage_in(ctx, ctx->scratch[0], rays, sizeof(MrtRay) * (size_t)n);
        if (st == MRT_OK) st = stage_in(ctx, ctx->scratch[2], dist, sizeof(float) * (size_t)n);
        if (st == MRT_OK) st = ensure(ctx, ctx->scratch[1], (size_t)n);
        if (st != MRT_OK) return st;
        d_rays = (const MrtRay *)ctx->scratch[0].ptr;
        d_dist = (const float *)ctx->scratch[2].ptr;
        d_occ = (uint8_t *)ctx->scratch[1].ptr;
    }
    st = launch_trace_any(s, d_rays, d_dist, n, d_occ);
    if (st == MRT_OK && mem == MRT_MEM_HOST)
        st = cuda_status(ctx, cudaMemcpyAsync(occluded, d_occ, (size_t)n, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
    if (st == MRT_OK) st = check_kernel_error(ctx);
    return st;
}

int mrt_trace_closest_counts(MrtScene *s, const MrtRay *rays, uint32_t n, uint32_t *node_fetch, uint32_t *tri_fetch,
                             uint32_t mem) {
    if (!s || (n && (!rays || !node_fetch || !tri_fetch))) return MRT_ERR_ARG;
    MrtContext *ctx = s->ctx;
    if (misaligned(ctx, mem, rays, 16, "rays") || misaligned(ctx, mem, node_fetch, 4, "node_fetch") ||
        misaligned(ctx, mem, tri_fetch, 4, "tri_fetch"))
        return MRT_ERR_ARG;
    if (!s->built) { set_error(ctx, "mrt_trace_closest_counts before mrt_scene_build"); return MRT_ERR_STATE; }
    if (!(s->opts.accelerator == MRT_ACCEL_BVH && s->opts.bvh_mode == MRT_BVH_FAST) &&
        s->opts.accelerator != MRT_ACCEL_REGULAR_GRID) {
        set_error(ctx, "mrt_trace_closest_counts: only the FAST BVH and the regular grid have a counting replay");
        return MRT_ERR_STATE;
    }
    if (n == 0) return MRT_OK;
    cudaSetDevice(ctx->device);
    const MrtRay *d_rays = rays;
    uint32_t *d_nodes = node_fetch, *d_tris = tri_fetch;
    int st = MRT_OK;
    if (mem == MRT_MEM_HOST) {
        st = stage_in(ctx, ctx->scratch[0], rays, sizeof(MrtRay) * (size_t)n);
        if (st == MRT_OK) st = ensure(ctx, ctx->scratch[1], 4ull * n);
        if (st == MRT_OK) st = ensure(ctx, ctx->scratch[2], 4ull * n);
        if (st != MRT_OK) return st;
        d_rays = (const MrtRay *)ctx->scratch[0].ptr;
        d_nodes = (uint32_t *)ctx->scratch[1].ptr;
        d_tris = (uint32_t *)ctx->scratch[2].ptr;
    }
    st = launch_trace_counts(s, d_rays, n, d_nodes, d_tris);
    if (st == MRT_OK && mem == MRT_MEM_HOST) {
        st = cuda_status(ctx, cudaMemcpyAsync(node_fetch, d_nodes, 4ull * n, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
        if (st == MRT_OK) st = cuda_status(ctx, cudaMemcpyAsync(tri_fetch, d_tris, 4ull * n, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
    }
    if (st == MRT_OK) st = check_kernel_error(ctx);
    return st;
}

}  // extern "C"
