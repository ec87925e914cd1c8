// mrt_wave.cuh - the per-ray pieces of the renderer shared by the single-frame render
// (mrt_render.cu) and the batch engine (mrt_batch.cu): task / pixel mapping, camera rays, light
// sampling, NoShadows shading, and the wavefront records with the shade and resolve steps of
// Whitted / PathTracer.
#pragma once

#include "mrt_persistent.cuh"

namespace mrt {

struct Task {
    uint32_t x, y, index;
};

struct RenderParams {
    DevCamera cam;
    uint32_t width, height, spp, spl, stride_px;
    int32_t pixel_sampler, light_sampler, rr_sampler, shader;
    float constant_value;
    int32_t depth_min, depth_max;
    uint64_t seed;
    uint32_t spp_offset;
    uint32_t strata;       // spp of the whole render (Stratified sampler strata)
    uint32_t task_base;    // first task of the current round (wavefront)
    // tasks: implicit rectangle (tasks == nullptr: x = t % width, y = t / width) or explicit list
    const Task *tasks;
    uint32_t n_tasks;
    uint32_t *bitmap;
    float4 *accum;
    float inv_w, inv_h, pw, ph;
    V3 depth_point;        // DepthMap maxPoint
};

// the shaders without secondary rays: the value is final at the camera ray
MRT_HD bool direct_shader(int shader) {
    return shader == MRT_SHADER_NOSHADOWS || shader == MRT_SHADER_DEPTHMAP || shader == MRT_SHADER_DIFFUSE;
}

__device__ __forceinline__ Task task_of(const RenderParams &p, uint32_t t) {
    if (p.tasks) return p.tasks[t];
    Task k;
    k.x = t % p.width;
    k.y = t / p.width;
    k.index = k.y * p.stride_px + k.x;
    return k;
}

// fp32 sum slot of the bitmap pixel a task writes (a task past the right edge wraps into the next
// row, as pixelIndex = y * stride + x does in Renderer.cpp:105); -1 when it lands in the row padding
__device__ __forceinline__ int64_t accum_slot(const RenderParams &p, const Task &k) {
    const uint32_t row = k.index / p.stride_px, col = k.index - row * p.stride_px;
    return col < p.width ? (int64_t)row * p.width + col : -1;
}

__device__ __forceinline__ Ray primary_ray(const RenderParams &p, const Task &k, const Stream &st) {
    const float u = (float)k.x * p.inv_w, v = (float)k.y * p.inv_h;   // Renderer.cpp:95-99
    const float r1 = draw(st, p.pixel_sampler, 0u, 0u);
    const float r2 = draw(st, p.pixel_sampler, 0u, 1u);
    return camera_ray(p.cam, u, v, (r1 - 0.5f) * 2.0f * p.pw, (r2 - 0.5f) * 2.0f * p.ph);
}

// Shader::getLight (Shader.cpp:225-236) and Light::getPosition (PointLight.cpp:17-19,
// AreaLight.cpp:22-31) for light sample j of a node
__device__ __forceinline__ const DevLight &pick_light(const DevScene &s, const Stream &st, uint32_t node, uint32_t j) {
    const float u = key_float(st.base, node, kDimLight + 3u * j);
    const uint32_t k = (uint32_t)floorf(u * (float)s.n_light * 0.99999f);
    return s.lights[k];
}
__device__ __forceinline__ V3 light_position(const DevLight &l, const Stream &st, int kind, uint32_t node, uint32_t j) {
    if (l.kind != MRT_LIGHT_AREA) return l.pos;
    float R = draw(st, kind, node, kDimLight + 3u * j + 1u);
    float S = draw(st, kind, node, kDimLight + 3u * j + 2u);
    if (R + S >= 1.0f) { R = 1.0f - R; S = 1.0f - S; }
    return (l.a + l.ab * R) + l.ac * S;
}

__device__ __forceinline__ bool material_of(const DevScene &s, const Isect &it, DevMaterial &m) {
    if (it.light >= 0) { m = s.lights[it.light].radiance; return true; }
    if (it.mat >= 0) { m = s.mats[it.mat]; return true; }
    return false;
}

// NoShadows::shade, NoShadows.cpp:19-65
__device__ __forceinline__ V3 shade_noshadows(const DevScene &s, const RenderParams &p, const Stream &st, const Isect &it,
                                              uint32_t node) {
    V3 rgb{0.0f, 0.0f, 0.0f};
    V3 kd;
    DevMaterial m;
    if (material_of(s, it, m)) {
        if (any_pos(m.le)) return m.le;
        kd = m.kd;
    } else {
        kd = it.color;
    }
    if (any_pos(kd) && s.n_light > 0) {
        for (uint32_t j = 0; j < p.spl; ++j) {
            const DevLight &l = pick_light(s, st, node, j);
            const V3 lp = light_position(l, st, p.light_sampler, node, j);
            const V3 vtl = normalize(lp - it.point);
            const float c = dot(it.normal, vtl);
            if (c > 0.0f) rgb = rgb + l.radiance.le * c;
        }
        rgb = rgb * kd;
        rgb = rgb / (float)p.spl;
    }
    return rgb + kd * 0.1f;
}

// DepthMap::shade, DepthMap.cpp:19-26
__device__ __forceinline__ V3 shade_depthmap(const RenderParams &p, const Ray &r, const Isect &it) {
    const float max_dist = length(p.depth_point - r.o) * 2.0f;
    const float x = (max_dist - it.length) / max_dist;
    const float depth = x < 0.0f ? 0.0f : x;   // std::max(x, 0)
    return V3{depth, depth, depth};
}

// DiffuseMaterial::shade, DiffuseMaterial.cpp:16-38
__device__ __forceinline__ V3 shade_diffuse(const DevScene &s, const Isect &it) {
    DevMaterial m;
    if (!material_of(s, it, m)) return it.color;
    if (any_pos(m.kd)) return m.kd;
    if (any_pos(m.ks)) return m.ks;
    if (any_pos(m.kt)) return m.kt;
    if (any_pos(m.le)) return m.le;
    return V3{0.0f, 0.0f, 0.0f};
}

// the value of a camera ray's hit under NoShadows, DepthMap or DiffuseMaterial
__device__ __forceinline__ V3 shade_direct(const DevScene &s, const RenderParams &p, const Stream &st, const Ray &r,
                                           const Isect &it) {
    if (p.shader == MRT_SHADER_DEPTHMAP) return shade_depthmap(p, r, it);
    if (p.shader == MRT_SHADER_DIFFUSE) return shade_diffuse(s, it);
    return shade_noshadows(s, p, st, it, 1u);
}


// ============================== wavefront records =============================================
enum NodeKind : uint32_t { kMiss = 0, kEmit = 1, kCut = 2, kShaded = 3 };
enum NodeFlag : uint32_t { kHasIndirect = 4, kRRScaled = 8, kKdPos = 16, kKsPos = 32, kKtPos = 64 };

struct RayRec {          // 48 bytes
    float ox, oy, oz, dx, dy, dz;
    int32_t depth;
    uint32_t exclude;
    uint32_t root;       // wave-local root index
    uint32_t parent;     // node index of the parent (0xFFFFFFFF for camera rays)
    uint32_t slot;       // 0 indirect, 1 specular, 2 transmission
    uint32_t code;       // path-tree code keying the stream (root 1, child code*4 + slot + 1)
};

struct NodeRec {         // 128 bytes
    uint32_t flags;      // kind | NodeFlag
    uint32_t occluded;   // bit j: shadow ray of light sample j was blocked
    float hit_t;
    uint32_t hit_id;
    V3 kd, ks, kt;       // 36
    V3 point, normal;    // 24 (or rgb of an emitter in `point`)
    V3 child[3];         // 36
    uint32_t child_flag; // bit s: child s reported a light hit
    uint32_t pad[3];
};

struct ShadowRec {       // 40 bytes
    float ox, oy, oz, dx, dy, dz, dist;
    uint32_t node;
    uint32_t j;
    uint32_t exclude;
};

struct Level {
    uint32_t start;
    uint32_t count;
    uint32_t shadow_count;
    uint32_t pad;
};

struct WaveState {
    RayRec *rays;
    NodeRec *nodes;
    ShadowRec *shadows;
    Level *levels;           // [max_levels + 1]
    float4 *root_rgb;        // per wave root: rgb, flag
    uint32_t ray_cap;
    uint32_t shadow_cap;
    uint32_t root_first;     // global index of the wave's first root
    uint32_t n_roots;
    unsigned long long *counters;   // [0] closest rays, [1] shadow rays
    // per-material shade queues: the shade kernel sorts each window of a level's rays by shading
    // class before shading them (scenes that mix diffuse with mirror / glass materials)
    uint32_t sort_shading;
};

// shading class of a ray after its closest hit: 0 nothing to shade here (a miss, a ray beyond the
// depth limit, an emitter), 1 diffuse only (light samples and the hemisphere ray), 2 a specular
// or transmitting material (mirror / refraction rays, Whitted.cpp:85-104, PathTracer.cpp:136-157)
constexpr int kShadeClasses = 3;
__device__ __forceinline__ uint32_t shade_class(const DevScene &s, const RenderParams &p, const RayRec &rr, uint32_t hit_id) {
    if (hit_id == MRT_HIT_NONE || rr.depth > p.depth_max) return 0u;
    const uint32_t type = MRT_HIT_TYPE(hit_id), i = MRT_HIT_INDEX(hit_id);
    int32_t m = -1;
    if (type == MRT_PRIM_TRIANGLE) m = s.tri_mat[i];
    else if (type == MRT_PRIM_SPHERE) m = s.sph_mat[i];
    else if (type == MRT_PRIM_PLANE) m = s.pln_mat[i];
    else return 0u;   // an area light: an emitter
    if (m < 0 || (uint32_t)m >= s.n_mat) return 1u;   // the primitive's colour: diffuse
    const DevMaterial &mt = s.mats[m];
    if (any_pos(mt.le)) return 0u;
    return (any_pos(mt.ks) || any_pos(mt.kt)) ? 2u : 1u;
}

__device__ __forceinline__ uint32_t warp_alloc(uint32_t want, uint32_t *counter) {
    // warp-aggregated allocation: inclusive scan of `want` across the warp, one atomic per warp.
    // Every lane of the warp calls this (the shade loop runs whole warps).
    __syncwarp();
    const int lane = threadIdx.x & 31;
    uint32_t incl = want;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += v;
    }
    uint32_t base = 0;
    if (lane == 31 && incl > 0) base = atomicAdd(counter, incl);
    base = __shfl_sync(0xFFFFFFFFu, base, 31);
    return base + incl - want;
}

__device__ __forceinline__ void root_task(const RenderParams &p, const WaveState &w, uint32_t root, Task &k,
                                          uint32_t &pixel, uint32_t &sample) {
    const uint32_t g = w.root_first + root;
    const uint32_t t = p.task_base + g / p.spp, si = g % p.spp;
    k = task_of(p, t);
    pixel = k.y * p.width + k.x;
    sample = p.spp_offset + si;
}


__device__ __forceinline__ Ray ray_of(const RayRec &r) {
    Ray x;
    x.o = V3{r.ox, r.oy, r.oz};
    x.d = V3{r.dx, r.dy, r.dz};
    x.depth = r.depth;
    x.exclude = r.exclude;
    return x;
}

__device__ __forceinline__ Level clamp_level(const WaveState &w, Level L) {
    // a level never reaches past the ray pool (overflowing children were dropped with MRT_ERR_LIMIT)
    L.start = min(L.start, w.ray_cap);
    L.count = min(L.count, w.ray_cap - L.start);
    return L;
}


// ---------------------------------------------------------------------------------------------
// per-ray pieces of the wavefront, shared by the single render and the batch
// ---------------------------------------------------------------------------------------------
struct ShadeLane {
    NodeRec nd;
    uint32_t child_mask;   // continuation rays: bit 0 indirect, 1 specular, 2 transmission
    uint32_t n_child;
    uint32_t n_shadow;
    bool shaded;
    uint32_t prim;         // Isect::prim: excluded from the continuation and shadow rays
    float ior;
};

// the part of Whitted::shade / PathTracer::shade before their recursive calls
// (Whitted.cpp:17-104, PathTracer.cpp:25-157): the node's own terms, its shadow-ray count and
// its continuation rays
__device__ __forceinline__ void shade_ray(const DevScene &s, const RenderParams &p, const RayRec &rr, uint32_t hit_id,
                                          float hit_t, const Stream &st, ShadeLane &o) {
    const Ray r = ray_of(rr);
    NodeRec &nd = o.nd;
    o.n_child = 0;
    o.n_shadow = 0;
    o.shaded = false;
    nd.flags = kMiss;
    nd.occluded = 0;
    nd.child_flag = 0;
    nd.child[0] = nd.child[1] = nd.child[2] = V3{0, 0, 0};
    nd.kd = nd.ks = nd.kt = V3{0, 0, 0};
    nd.point = nd.normal = V3{0, 0, 0};
    nd.hit_id = hit_id;
    nd.hit_t = hit_t;
    o.child_mask = 0;
    Isect isect;
    if (hit_id == MRT_HIT_NONE || !make_isect(s, r, hit_id, isect)) return;
    if (r.depth > p.depth_max) {
        nd.flags = kCut;   // Whitted.cpp:20-22, PathTracer.cpp:28-31
        return;
    }
    DevMaterial m;
    V3 kd, ks{0, 0, 0}, kt{0, 0, 0};
    float ior = 1.0f;
    if (material_of(s, isect, m)) {
        if (any_pos(m.le)) { nd.flags = kEmit; nd.point = m.le; return; }
        kd = m.kd; ks = m.ks; kt = m.kt; ior = m.ior;
    } else {
        kd = isect.color;
    }
    o.shaded = true;
    nd.flags = kShaded;
    nd.kd = kd; nd.ks = ks; nd.kt = kt;
    nd.point = isect.point;
    nd.normal = isect.normal;
    const bool kd_pos = any_pos(kd), ks_pos = any_pos(ks), kt_pos = any_pos(kt);
    if (kd_pos) nd.flags |= kKdPos;
    if (ks_pos) nd.flags |= kKsPos;
    if (kt_pos) nd.flags |= kKtPos;
    if (kd_pos && s.n_light > 0) {
        for (uint32_t j = 0; j < p.spl; ++j) {
            const DevLight &l = pick_light(s, st, rr.code, j);
            const V3 lp = light_position(l, st, p.light_sampler, rr.code, j);
            const V3 vtl = normalize(lp - isect.point);
            if (dot(isect.normal, vtl) > 0.0f) ++o.n_shadow;
        }
    }
    if (p.shader == MRT_SHADER_PATHTRACER && kd_pos) {
        bool go = r.depth <= p.depth_min;   // PathTracer.cpp:106-107
        if (!go) go = draw(st, p.rr_sampler, rr.code, kDimRR) > 0.5f;
        if (go) {
            nd.flags |= kHasIndirect;
            if (r.depth > p.depth_min) nd.flags |= kRRScaled;
            o.child_mask |= 1u;
        }
    }
    if (ks_pos) o.child_mask |= 2u;
    if (kt_pos) o.child_mask |= 4u;
    o.n_child = __popc(o.child_mask);
    o.prim = isect.prim;
    o.ior = ior;
}

// the node record as the resolve pass reads it: a miss or a cut node only its flags, an emitter
// its radiance, a shaded node its terms with the occlusion and child-flag bits cleared (the
// children's values arrive from their own resolve)
__device__ __forceinline__ void store_node(NodeRec &dst, const NodeRec &nd) {
    dst.flags = nd.flags;
    const uint32_t kind = nd.flags & 3u;
    if (kind == kEmit) dst.point = nd.point;
    if (kind != kShaded) return;
    dst.occluded = 0;
    dst.child_flag = 0;
    dst.kd = nd.kd;
    dst.ks = nd.ks;
    dst.kt = nd.kt;
    dst.point = nd.point;
    dst.normal = nd.normal;
}

// the direction of the continuation ray of `slot` from a shaded node (the hemisphere sample of the
// indirect ray, PathTracer.cpp:106-134; mirror and refraction, Whitted.cpp:85-104,
// PathTracer.cpp:136-157); d = the incoming direction, code = the node's path-tree code
__device__ __forceinline__ V3 child_dir(const ShadeLane &o, const V3 &d, const Stream &st, uint32_t code, uint32_t slot) {
    if (slot == 0u) return hemisphere(o.nd.normal, key_float(st.base, code, kDimHemi), key_float(st.base, code, kDimHemi + 1u));
    if (slot == 1u) return reflect(d, o.nd.normal);
    return refract(d, o.nd.normal, 1.0f / o.ior);
}

// the continuation rays in slot order, from the hit point
__device__ __forceinline__ void emit_children(const DevScene &s, const ShadeLane &o, const RayRec &rr, const Stream &st,
                                              uint32_t idx, uint32_t pos0, RayRec *rays, uint32_t cap) {
    const V3 d{rr.dx, rr.dy, rr.dz};
    uint32_t pos = pos0;
    for (uint32_t m = o.child_mask; m; m &= m - 1u) {
        const uint32_t slot = (uint32_t)(__ffs(m) - 1);
        if (pos >= cap) { raise_error(s, MRT_ERR_LIMIT); break; }
        const V3 cd = child_dir(o, d, st, rr.code, slot);
        RayRec q;
        q.ox = o.nd.point.x; q.oy = o.nd.point.y; q.oz = o.nd.point.z;
        q.dx = cd.x; q.dy = cd.y; q.dz = cd.z;
        q.depth = rr.depth + 1;
        q.exclude = o.prim;
        q.root = rr.root;
        q.parent = idx;
        q.slot = slot;
        q.code = rr.code * 4u + slot + 1u;
        rays[pos++] = q;
    }
}

// the shadow rays of light samples with cos > 0, in light-sample order (Whitted.cpp:33-66)
__device__ __forceinline__ void emit_shadows(const DevScene &s, const RenderParams &p, const Stream &st, const ShadeLane &o,
                                             const RayRec &rr, uint32_t idx, uint32_t pos0, ShadowRec *shadows,
                                             uint32_t cap) {
    if (!o.shaded || o.n_shadow == 0) return;
    uint32_t q = 0;
    for (uint32_t j = 0; j < p.spl; ++j) {
        const DevLight &l = pick_light(s, st, rr.code, j);
        const V3 lp = light_position(l, st, p.light_sampler, rr.code, j);
        V3 vtl = lp - o.nd.point;
        const float dist = length(vtl);
        vtl = normalize(vtl);
        if (!(dot(o.nd.normal, vtl) > 0.0f)) continue;
        const uint32_t pos = pos0 + q++;
        if (pos >= cap) { raise_error(s, MRT_ERR_LIMIT); break; }
        ShadowRec sr;
        sr.ox = o.nd.point.x; sr.oy = o.nd.point.y; sr.oz = o.nd.point.z;
        sr.dx = vtl.x; sr.dy = vtl.y; sr.dz = vtl.z;
        sr.dist = dist;
        sr.node = idx;
        sr.j = j;
        sr.exclude = o.prim;
        shadows[pos] = sr;
    }
}

// the rest of shade() once the children returned: Whitted.cpp:64-106, PathTracer.cpp:100-163
__device__ __forceinline__ void resolve_node(const DevScene &s, const RenderParams &p, const NodeRec &nd, const RayRec &rr,
                                             const Stream &st, V3 &rgb, bool &flag) {
    rgb = V3{0.0f, 0.0f, 0.0f};
    flag = false;
    const uint32_t kind = nd.flags & 3u;
    if (kind == kEmit) {
        rgb = nd.point;
        flag = true;
        return;
    }
    if (kind != kShaded) return;
    V3 direct{0.0f, 0.0f, 0.0f};
    const bool kd_pos = (nd.flags & kKdPos) != 0;
    if (kd_pos && s.n_light > 0) {
        for (uint32_t j = 0; j < p.spl; ++j) {
            const DevLight &l = pick_light(s, st, rr.code, j);
            const V3 lp = light_position(l, st, p.light_sampler, rr.code, j);
            const V3 vtl = normalize(lp - nd.point);
            const float c = dot(nd.normal, vtl);
            if (c > 0.0f && !((nd.occluded >> (j & 31u)) & 1u)) direct = direct + l.radiance.le * c;
        }
        direct = direct * nd.kd;
        direct = direct / (float)p.spl;
    }
    if (p.shader == MRT_SHADER_WHITTED) {   // Whitted.cpp:64-106
        rgb = direct;
        if (nd.flags & kKsPos) rgb = rgb + nd.ks * nd.child[1];
        if (nd.flags & kKtPos) rgb = rgb + nd.kt * nd.child[2];
        rgb = rgb + nd.kd * 0.1f;
        return;
    }
    V3 lid{0.0f, 0.0f, 0.0f}, lis{0.0f, 0.0f, 0.0f}, lit{0.0f, 0.0f, 0.0f};   // PathTracer.cpp:100-163
    if (nd.flags & kHasIndirect) {
        lid = lid + nd.kd * nd.child[0];
        if (nd.flags & kRRScaled) lid = lid / (0.5f * 0.5f);
        flag = (nd.child_flag & 1u) != 0;
        if (any_pos(direct) && flag) lid = V3{0.0f, 0.0f, 0.0f};
    }
    if (nd.flags & kKsPos) lis = lis + nd.ks * nd.child[1];
    if (nd.flags & kKtPos) lit = lit + nd.kt * nd.child[2];
    rgb = rgb + direct;
    rgb = rgb + lid;
    rgb = rgb + lis;
    rgb = rgb + lit;
}

}  // namespace mrt
