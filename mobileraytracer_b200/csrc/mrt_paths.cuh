// mrt_paths.cuh - Whitted / PathTracer camera paths traced whole, one path per lane, in one
// persistent launch.
//
// The wavefront (one kernel per bounce level for a wave of paths) waits at every level for its
// slowest ray: deep levels hold few rays and leave most of the GPU idle, and every level pays launch
// and queue traffic.  Here a lane takes a camera path, follows its shade() recursion depth first
// (Whitted.cpp:17-107, PathTracer.cpp:25-164) with the frames of the recursion in its own stack
// (local memory), and asks the traversal engine for one query at a time: the closest hit of the
// frame's ray, then its shadow rays (any hit), then its continuation rays in slot order; when a
// frame has all its answers it is resolved (resolve_node, the same arithmetic as the wavefront's
// bottom-up pass) into its parent, and the root's value goes to the wave's per-path slot for the
// sample-ordered fold.  Rays of different depths and kinds share the warp; the warp-voted node and
// leaf phases of the persistent engine keep the lanes together where they can.
//
// Results equal the wavefront's bit for bit: every query is answered exactly (closest = the
// lexicographic minimum (t, index) of the accepted hits, any = the reference's occlusion test), and
// the per-node arithmetic is the shared shade_ray / resolve_node of mrt_wave.cuh, keyed by the same
// path-tree codes.
#pragma once

#include "mrt_wave.cuh"

namespace mrt {

constexpr int kPathFrames = 12;   // recursion depth a lane can hold: depth_max + 1 <= kPathFrames

struct PathFrame {
    NodeRec nd;           // the node's own terms, then its children's values
    uint32_t code;        // path-tree code
    int32_t depth;
    uint32_t slot;        // slot in the parent
    uint8_t n_child, next_child, next_j, shaded;
    V3 child_d[3];        // continuation directions (origin = the hit point)
    uint8_t child_slot[3];
    uint8_t pad;
};

// the lane's side of a path: its frames, the sample it belongs to and its query counts
struct PathLane {
    PathFrame fr[kPathFrames];
    int top;              // frames in use
    uint32_t item;        // work item (wave path index)
    uint32_t job;
    FastView v;           // the job scene's tree (batched jobs)
    Stream st;
    uint32_t n_closest, n_shadow;
};

// shadow ray of light sample j of a shaded node (Whitted.cpp:33-66: light position, direction,
// distance, the cos > 0 test); false when the sample is skipped
__device__ __forceinline__ bool shadow_query(const DevScene &s, const RenderParams &p, const Stream &st,
                                             const PathFrame &f, uint32_t j, Ray &r, float &dist) {
    const DevLight &l = pick_light(s, st, f.code, j);
    const V3 lp = light_position(l, st, p.light_sampler, f.code, j);
    V3 vtl = lp - f.nd.point;
    dist = length(vtl);
    vtl = normalize(vtl);
    if (!(dot(f.nd.normal, vtl) > 0.0f)) return false;
    r.o = f.nd.point;
    r.d = vtl;
    r.depth = 0;
    r.exclude = MRT_HIT_TYPE(f.nd.hit_id) == MRT_PRIM_SPHERE ? MRT_HIT_NONE : f.nd.hit_id;   // Isect::prim
    return true;
}

// After the closest hit of the top frame's ray: the node's own terms (shade_ray) and its children.
__device__ __forceinline__ void path_shade(const DevScene &s, const RenderParams &p, PathLane &L, const Ray &r,
                                           uint32_t hit_id, float hit_t) {
    PathFrame &f = L.fr[L.top - 1];
    RayRec rr;
    rr.ox = r.o.x; rr.oy = r.o.y; rr.oz = r.o.z;
    rr.dx = r.d.x; rr.dy = r.d.y; rr.dz = r.d.z;
    rr.depth = f.depth;
    rr.exclude = r.exclude;
    rr.root = 0;
    rr.parent = 0;
    rr.slot = f.slot;
    rr.code = f.code;
    ShadeLane o;
    if (direct_shader(p.shader)) {
        // NoShadows / DepthMap / DiffuseMaterial: the value is final at the camera ray
        o.n_child = 0;
        o.child_mask = 0;
        o.shaded = false;
        NodeRec &nd = o.nd;
        nd.flags = kMiss;
        nd.occluded = 0;
        nd.child_flag = 0;
        nd.hit_id = hit_id;
        nd.hit_t = hit_t;
        nd.point = V3{0, 0, 0};
        Isect it;
        if (hit_id != MRT_HIT_NONE && make_isect(s, r, hit_id, it)) {
            nd.flags = kEmit;
            nd.point = shade_direct(s, p, L.st, r, it);
        }
    } else {
        shade_ray(s, p, rr, hit_id, hit_t, L.st, o);
    }
    f.nd = o.nd;
    f.shaded = o.shaded && (o.nd.flags & kKdPos) && s.n_light > 0 ? 1 : 0;
    f.n_child = (uint8_t)o.n_child;
    f.next_child = 0;
    f.next_j = 0;
    uint32_t c = 0;
    for (uint32_t m = o.child_mask; m; m &= m - 1u, ++c) {
        const uint32_t slot = (uint32_t)(__ffs(m) - 1);
        f.child_d[c] = child_dir(o, r.d, L.st, f.code, slot);
        f.child_slot[c] = (uint8_t)slot;
    }
}

// The lane's next query, resolving finished frames into their parents on the way.  Returns false
// when the path's root is resolved (its value in rgb, flag).
__device__ __forceinline__ bool path_next(const DevScene &s, const RenderParams &p, PathLane &L, Ray &r, float &dist,
                                          bool &any, V3 &rgb, bool &flag) {
    for (int guard = 0; guard < 4 * kPathFrames + 64; ++guard) {
        PathFrame &f = L.fr[L.top - 1];
        while (f.shaded && f.next_j < p.spl) {   // shadow rays first, in light-sample order
            const uint32_t j = f.next_j++;
            if (shadow_query(s, p, L.st, f, j, r, dist)) {
                any = true;
                return true;
            }
        }
        if (f.next_child < f.n_child) {          // then the continuation rays, in slot order
            const uint32_t c = f.next_child++;
            if (L.top >= kPathFrames) { raise_error(s, MRT_ERR_LIMIT); break; }
            PathFrame &g = L.fr[L.top++];
            g.code = f.code * 4u + f.child_slot[c] + 1u;
            g.depth = f.depth + 1;
            g.slot = f.child_slot[c];
            r.o = f.nd.point;
            r.d = f.child_d[c];
            r.depth = g.depth;
            r.exclude = MRT_HIT_TYPE(f.nd.hit_id) == MRT_PRIM_SPHERE ? MRT_HIT_NONE : f.nd.hit_id;
            dist = kRayLengthMax;
            any = false;
            return true;
        }
        // every answer is in: the rest of shade() (resolve_node) and up to the parent
        RayRec rr;
        rr.code = f.code;
        V3 v;
        bool fl;
        resolve_node(s, p, f.nd, rr, L.st, v, fl);
        const uint32_t slot = f.slot;
        --L.top;
        if (L.top == 0) {
            rgb = v;
            flag = fl;
            return false;
        }
        PathFrame &pf = L.fr[L.top - 1];
        pf.nd.child[slot] = v;
        if (fl) pf.nd.child_flag |= 1u << slot;
    }
    // unreachable for consistent frames: end the path with black
    L.top = 0;
    rgb = V3{0, 0, 0};
    flag = false;
    return false;
}

// Work provides: total(), counter(), scene(lane), view(lane), params(lane),
//   begin(item, lane, r): the path's camera ray (the lane's frames reset, root frame pushed),
//   deliver(lane, rgb, flag): the path's value.
template <class Work>
__device__ void persistent_paths(Work &work) {
    const uint32_t FULL = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const uint32_t total = work.total();
    bool active = false;
    bool exhausted = false;
    PathLane lane;
    lane.n_closest = 0;
    lane.n_shadow = 0;
    Ray r;
    float dist = kRayLengthMax;
    bool any = false;
    FastTrav t;
    TravStack stk;
    auto start = [&](const DevScene &s) {
        if (any) {
            ++lane.n_shadow;
            trav_begin<false>(s, r, dist, MRT_HIT_NONE, t);
            if (naive_occ<kPlane>(s, r, dist) || naive_occ<kSphere>(s, r, dist)) {
                trav_set_occluded(t);
                trav_clear(t);
            }
        } else {
            ++lane.n_closest;
            float len = kRayLengthMax;
            uint32_t id = MRT_HIT_NONE;
            naive_trace<kPlane>(s, r, len, id);
            naive_trace<kSphere>(s, r, len, id);
            trav_begin<false>(s, r, len, id, t);
        }
    };
    for (;;) {
        // 1. refill idle lanes (one atomic per warp)
        const uint32_t idle = __ballot_sync(FULL, !active);
        if (!exhausted && (__popc(idle) >= 8 || idle == FULL)) {
            const int leader = __ffs(idle) - 1;
            uint32_t base = 0;
            if (lane_id == leader) base = atomicAdd(work.counter(), (uint32_t)__popc(idle));
            base = __shfl_sync(FULL, base, leader);
            if (base + (uint32_t)__popc(idle) >= total) exhausted = true;
            if (!active) {
                const uint32_t item = base + __popc(idle & ((1u << lane_id) - 1u));
                if (item < total) {
                    work.begin(item, lane, r);
                    dist = kRayLengthMax;
                    any = false;
                    start(work.scene(lane));
                    active = true;
                }
            }
        }
        if (__ballot_sync(FULL, active) == 0) {
            if (exhausted) break;
            continue;
        }
        // 2. node phase
        for (;;) {   // lanes holding a leaf step on speculatively while others search
            const bool w = active && trav_wants_node(t);
            if (node_phase_over(w, active && trav_has_leaf(t))) break;
            if (w || (active && trav_can_speculate(t))) trav_node_step<false>(work.view(lane), r, t, stk);
        }
        // 3. leaf phase (an any-hit query ends at its first occluder)
        if (active && trav_has_leaf(t)) {
            if (any) trav_occ_leaf_step(work.view(lane), r, t);
            else trav_leaf_step<false>(work.view(lane), r, t);
        }
        // 4. completion: the answer moves the path on.  Lanes whose query is answered wait until
        // 24 of the warp's lanes (or all its active lanes) are, so the shading code runs with the
        // warp mostly converged
        const uint32_t fin = __ballot_sync(FULL, active && trav_finished(t)), act = __ballot_sync(FULL, active);
        if ((__popc(fin) >= 24 || fin == act) && active && trav_finished(t)) {
            const DevScene &s = work.scene(lane);
            const RenderParams &p = work.params(lane);
            if (any) {
                if (trav_hit(t)) {
                    PathFrame &f = lane.fr[lane.top - 1];
                    f.nd.occluded |= 1u << ((f.next_j - 1u) & 31u);
                }
            } else {
                float len = t.best_t;
                uint32_t id = t.best_id;
                const bool hit_light = lights_trace(s, r, len, id);
                const bool hit = id != MRT_HIT_NONE || hit_light;
                path_shade(s, p, lane, r, hit ? id : MRT_HIT_NONE, len);
            }
            V3 rgb;
            bool flag;
            if (path_next(s, p, lane, r, dist, any, rgb, flag)) {
                start(s);
            } else {
                work.deliver(lane, rgb, flag);
                active = false;
            }
        }
    }
    work.count(lane.n_closest, lane.n_shadow);
}

}  // namespace mrt
