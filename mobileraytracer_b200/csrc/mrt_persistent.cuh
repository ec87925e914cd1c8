// mrt_persistent.cuh - persistent closest-hit engine for the FAST BVH.
//
// Rays in a warp need very different amounts of work (a camera ray that misses the scene ends at
// the root box, one that crosses a dense soup visits ~60 node pairs), so a one-ray-per-thread
// kernel leaves most lanes idle behind the warp's longest ray.  Here every lane carries a
// resumable traversal state and the warp loops:
//   1. refill: lanes whose work item is finished take new items from a global counter, one
//      atomicAdd per warp for all of them (ballot + popc);
//   2. node phase: lanes that have no pending leaf expand 4-wide nodes until fewer than
//      kNodeQuorum lanes still search (warp vote), so node visits of different lanes run
//      together; lanes holding one leaf go on speculatively up to a second one;
//   3. leaf phase: pending leaves are intersected together;
//   4. completion: finished rays hand their result to the work item, which may start its next
//      ray in the same lane (e.g. the next sample of a pixel).
// Semantics are those of fast_trace(): the result is the lexicographic minimum (t, index) of the
// triangles passing the reference test below the incoming length.
#pragma once

#include "mrt_trace.cuh"

namespace mrt {

struct FastTrav {
    FastRay f;
    float best_t;
    uint32_t best_i;
    uint32_t node;          // node to expand next (kNodeNone: pop the stack)
    uint32_t leaf_first, leaf_count;   // pending leaf (count 0: none)
    uint32_t leaf2_first, leaf2_count; // a second leaf found while waiting for the warp (speculative)
    int sp;
    bool have;
    uint32_t c_nodes, c_tris;
};

// the traversal stack lives apart from the scalar state so the scalars stay in registers.  It holds
// node and leaf codes only: a popped entry is not culled by its entry distance (the children of a
// popped node still meet the box test against the best distance).  Keeping the distances and
// culling at the pop cost one more local load and store per entry and was 8 % slower on the
// 1,000,000-triangle soup frame than expanding the few entries it would have culled.
struct TravStack {
    uint32_t n[kFastStack];
};

template <bool kCount>
__device__ __forceinline__ void trav_begin(const DevScene &s, const Ray &r, float len0, FastTrav &t) {
    t.f = fast_ray(r);
    t.best_t = len0;
    t.best_i = 0;
    t.have = false;
    t.node = s.n_tri == 0 ? kNodeNone : 0u;   // the root node
    t.leaf_count = 0;
    t.leaf2_count = 0;
    t.sp = 0;
    t.c_nodes = 0;
    t.c_tris = 0;
}

__device__ __forceinline__ bool trav_wants_node(const FastTrav &t) {
    return t.leaf_count == 0 && (t.node != kNodeNone || t.sp > 0);
}
// a lane with one pending leaf may go on with node steps while others of its warp still search
// (Aila and Laine, "Understanding the efficiency of ray traversal on GPUs", HPG 2009: speculative
// traversal), up to a second leaf
__device__ __forceinline__ bool trav_can_speculate(const FastTrav &t) {
    return t.leaf_count > 0 && t.leaf2_count == 0 && (t.node != kNodeNone || t.sp > 0);
}
__device__ __forceinline__ bool trav_finished(const FastTrav &t) {
    return t.leaf_count == 0 && t.leaf2_count == 0 && t.node == kNodeNone && t.sp == 0;
}

// the node phase of a warp ends when no lane searches any more, or when fewer than kNodeQuorum lanes
// search while others hold leaves: those leaves are tested first, and the few searching lanes go on
// in the next node phase (2 and 4: +2 % on the 1,000,000-triangle soup frame, 8: -2 %)
constexpr int kNodeQuorum = 4;
__device__ __forceinline__ bool node_phase_over(bool searching, bool holding_leaf) {
    const uint32_t s = __ballot_sync(0xFFFFFFFFu, searching);
    return s == 0u || (__popc(s) < kNodeQuorum && __any_sync(0xFFFFFFFFu, holding_leaf));
}

__device__ __forceinline__ void trav_take(FastTrav &t, uint32_t code) {
    if (code & kLeafCode) {
        if (t.leaf_count == 0) {
            t.leaf_first = code_first(code);
            t.leaf_count = code_count(code);
        } else {
            t.leaf2_first = code_first(code);
            t.leaf2_count = code_count(code);
        }
        t.node = kNodeNone;
    } else {
        t.node = code;
    }
}

// one node step: expand the current node (popping one first when there is none), nearest child
// next and the other hits pushed far to near
template <bool kCount, class S>
__device__ __forceinline__ void trav_node_step(const S &s, FastTrav &t, TravStack &st) {
    if (t.node == kNodeNone) {
        if (t.sp > 0) { --t.sp; trav_take(t, st.n[t.sp]); }
        if (t.node == kNodeNone) return;   // a leaf, or nothing left
    }
    if (!node_in_range(s, t.node)) { raise_error(s, MRT_ERR_LIMIT); t.node = kNodeNone; t.sp = 0; return; }
    float ct[kWide];
    uint32_t cc[kWide];
    const int n = wide_children<true>(s, t.node, t.f, t.best_t, ct, cc);
    if (kCount) t.c_nodes += kWide;
    t.node = kNodeNone;
    if (n == 0) return;
    if (t.sp + n - 1 > kFastStack) { raise_error(s, MRT_ERR_LIMIT); t.sp = 0; return; }
#pragma unroll
    for (int k = kWide - 1; k >= 1; --k)
        if (k < n) { st.n[t.sp] = cc[k]; ++t.sp; }
    trav_take(t, cc[0]);
}

template <bool kCount, class S>
__device__ __forceinline__ void trav_leaf_step(const S &s, const Ray &r, FastTrav &t) {
    FastCounts cnt{0, 0};
    fast_leaf<kCount>(s, r, t.leaf_first, t.leaf_count, t.best_t, t.best_i, t.have, cnt);
    if (t.leaf2_count) fast_leaf<kCount>(s, r, t.leaf2_first, t.leaf2_count, t.best_t, t.best_i, t.have, cnt);
    if (kCount) t.c_tris += cnt.tris;
    t.leaf_count = 0;
    t.leaf2_count = 0;
}

// ---------------------------------------------------------------------------------------------
// the persistent loop.  Work provides:
//   uint32_t total() const; uint32_t *counter() const;
//   const DevScene &scene(const Lane &lane, const DevScene &s) -> the scene the lane's ray is
//        traced in (s itself for a single-scene launch; the lane's job scene in a batch)
//   view(lane, s) -> what the node and leaf steps read of that scene (s itself, or a FastView
//        the lane keeps in registers)
//   bool begin(uint32_t item, Lane &lane, Ray &r)     -> false: nothing to trace for this item
//   bool finish(Lane &lane, Ray &r, bool hit, float t, uint32_t id, const FastTrav &tr)
//        -> true: r holds the item's next ray (same lane continues)
// Planes and spheres are tested in order before the tree and area lights after it
// (Shader.cpp:124-150), all with the reference accept rule.
// ---------------------------------------------------------------------------------------------
template <bool kCount, class Work, class Lane>
__device__ __forceinline__ void start_ray(const DevScene &s, const Ray &r, FastTrav &t, float &len, uint32_t &id) {
    len = kRayLengthMax;
    id = MRT_HIT_NONE;
    naive_trace<kPlane>(s, r, len, id);
    naive_trace<kSphere>(s, r, len, id);
    trav_begin<kCount>(s, r, len, t);
}

template <bool kCount, class Work, class Lane>
__device__ void persistent_closest(const DevScene &s, Work &work, Lane &lane) {
    const uint32_t FULL = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const uint32_t total = work.total();
    bool active = false;
    bool exhausted = false;
    Ray r;
    FastTrav t;
    TravStack stk;
    float len0 = kRayLengthMax;   // distance after planes and spheres
    uint32_t id0 = MRT_HIT_NONE;
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
                if (item < total && work.begin(item, lane, r)) {
                    start_ray<kCount, Work, Lane>(work.scene(lane, s), r, t, len0, id0);
                    active = true;
                }
            }
        }
        if (__ballot_sync(FULL, active) == 0) {
            if (exhausted) break;
            continue;
        }
        // 2. node phase (lanes holding a leaf step on speculatively while others search)
        for (;;) {
            const bool w = active && trav_wants_node(t);
            if (node_phase_over(w, active && t.leaf_count > 0)) break;
            if (w || (active && trav_can_speculate(t))) trav_node_step<kCount>(work.view(lane, s), t, stk);
        }
        // 3. leaf phase
        if (active && t.leaf_count > 0) trav_leaf_step<kCount>(work.view(lane, s), r, t);
        // 4. completion
        if (active && trav_finished(t)) {
            float len = len0;
            uint32_t id = id0;
            if (t.have) { len = t.best_t; id = hid(MRT_PRIM_TRIANGLE, t.best_i); }
            const bool hit_light = lights_trace(work.scene(lane, s), r, len, id);
            const bool hit = id != MRT_HIT_NONE || hit_light;
            if (work.finish(lane, r, hit, len, id, t)) start_ray<kCount, Work, Lane>(work.scene(lane, s), r, t, len0, id0);
            else active = false;
        }
    }
}

}  // namespace mrt

namespace mrt {

// ---------------------------------------------------------------------------------------------
// any-hit (Shader::shadowTrace, Shader.cpp:162-187): planes and spheres in order, then the tree;
// the first occluder ends the ray, so no ordering and no distance culling beyond `dist`.
// Work provides total(), counter(), scene(lane, s), begin(item, lane, r, dist) and finish(lane, occluded).
// ---------------------------------------------------------------------------------------------
struct OccTrav {
    FastRay f;
    float dist;
    uint32_t node;
    uint32_t leaf_first, leaf_count;
    uint32_t leaf2_first, leaf2_count;   // speculative second leaf
    int sp;
    bool occluded;
};

__device__ __forceinline__ void occ_begin(const DevScene &s, const Ray &r, float dist, OccTrav &t) {
    t.dist = dist;
    t.node = kNodeNone;
    t.leaf_count = 0;
    t.leaf2_count = 0;
    t.sp = 0;
    t.occluded = naive_occ<kPlane>(s, r, dist) || naive_occ<kSphere>(s, r, dist);
    if (t.occluded || s.n_tri == 0) return;
    t.f = fast_ray(r);
    t.node = 0u;
}

__device__ __forceinline__ bool occ_wants_node(const OccTrav &t) {
    return !t.occluded && t.leaf_count == 0 && (t.node != kNodeNone || t.sp > 0);
}
__device__ __forceinline__ bool occ_can_speculate(const OccTrav &t) {
    return !t.occluded && t.leaf_count > 0 && t.leaf2_count == 0 && (t.node != kNodeNone || t.sp > 0);
}
__device__ __forceinline__ bool occ_finished(const OccTrav &t) {
    return t.occluded || (t.leaf_count == 0 && t.leaf2_count == 0 && t.node == kNodeNone && t.sp == 0);
}

__device__ __forceinline__ void occ_take(OccTrav &t, uint32_t code) {
    if (code & kLeafCode) {
        if (t.leaf_count == 0) {
            t.leaf_first = code_first(code);
            t.leaf_count = code_count(code);
        } else {
            t.leaf2_first = code_first(code);
            t.leaf2_count = code_count(code);
        }
        t.node = kNodeNone;
    } else {
        t.node = code;
    }
}

template <class S>
__device__ __forceinline__ void occ_node_step(const S &s, OccTrav &t, uint32_t *stack_n) {
    if (t.node == kNodeNone) {
        if (t.sp > 0) occ_take(t, stack_n[--t.sp]);
        if (t.node == kNodeNone) return;   // a leaf, or nothing left
    }
    if (!node_in_range(s, t.node)) { raise_error(s, MRT_ERR_LIMIT); t.node = kNodeNone; t.sp = 0; return; }
    float ct[kWide];
    uint32_t cc[kWide];
    const int n = wide_children<false>(s, t.node, t.f, t.dist, ct, cc);
    t.node = kNodeNone;
    if (n == 0) return;
    if (t.sp + n - 1 > kFastStack) { raise_error(s, MRT_ERR_LIMIT); t.sp = 0; return; }
#pragma unroll
    for (int k = kWide - 1; k >= 1; --k)
        if (k < n) stack_n[t.sp++] = cc[k];
    occ_take(t, cc[0]);
}

template <class S>
__device__ __forceinline__ void occ_leaf_step(const S &s, const Ray &r, OccTrav &t) {
    for (int q = 0; q < 2 && !t.occluded; ++q) {
        const uint32_t first = q == 0 ? t.leaf_first : t.leaf2_first, count = q == 0 ? t.leaf_count : t.leaf2_count;
        if (count == 0) continue;
        if (first + count > s.n_tri) { raise_error(s, MRT_ERR_LIMIT); break; }
        for (uint32_t k = first; k < first + count; ++k) {
            const float4 A = __ldg(&s.ftris[3 * k]);
            const float4 AB = __ldg(&s.ftris[3 * k + 1]);
            const float4 AC = __ldg(&s.ftris[3 * k + 2]);
            if (r.exclude == hid(MRT_PRIM_TRIANGLE, __float_as_uint(A.w))) continue;
            if (tri_occ(v3(A), v3(AB), v3(AC), r, t.dist)) { t.occluded = true; break; }
        }
    }
    t.leaf_count = 0;
    t.leaf2_count = 0;
}

template <class Work, class Lane>
__device__ void persistent_any(const DevScene &s, Work &work, Lane &lane) {
    const uint32_t FULL = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const uint32_t total = work.total();
    bool active = false;
    bool exhausted = false;
    Ray r;
    OccTrav t;
    uint32_t stack_n[kFastStack];
    for (;;) {
        const uint32_t idle = __ballot_sync(FULL, !active);
        if (!exhausted && (__popc(idle) >= 8 || idle == FULL)) {
            const int leader = __ffs(idle) - 1;
            uint32_t base = 0;
            if (lane_id == leader) base = atomicAdd(work.counter(), (uint32_t)__popc(idle));
            base = __shfl_sync(FULL, base, leader);
            if (base + (uint32_t)__popc(idle) >= total) exhausted = true;
            if (!active) {
                const uint32_t item = base + __popc(idle & ((1u << lane_id) - 1u));
                float dist;
                if (item < total && work.begin(item, lane, r, dist)) {
                    occ_begin(work.scene(lane, s), r, dist, t);
                    active = true;
                }
            }
        }
        if (__ballot_sync(FULL, active) == 0) {
            if (exhausted) break;
            continue;
        }
        for (;;) {
            const bool w = active && occ_wants_node(t);
            if (node_phase_over(w, active && t.leaf_count > 0)) break;
            if (w || (active && occ_can_speculate(t))) occ_node_step(work.view(lane, s), t, stack_n);
        }
        if (active && t.leaf_count > 0) occ_leaf_step(work.view(lane, s), r, t);
        if (active && occ_finished(t)) {
            work.finish(lane, t.occluded);
            active = false;
        }
    }
}

}  // namespace mrt
