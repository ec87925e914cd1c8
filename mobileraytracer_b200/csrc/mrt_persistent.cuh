// mrt_persistent.cuh - persistent closest-hit engine for the FAST BVH.
//
// Rays in a warp need very different amounts of work (a camera ray that misses the scene ends at
// the root box, one that crosses a dense soup visits ~60 node pairs), so a one-ray-per-thread
// kernel leaves most lanes idle behind the warp's longest ray.  Here every lane carries a
// resumable traversal state and the warp loops:
//   1. refill: lanes whose work item is finished take new items from a global counter, one
//      atomicAdd per warp for all of them (ballot + popc);
//   2. node phase: lanes that have no triangles waiting expand 8-wide nodes until fewer than
//      kNodeQuorum lanes still search (warp vote), so node visits of different lanes run
//      together; lanes holding triangles go on speculatively up to a second group of them;
//   3. leaf phase: the waiting triangles are intersected together;
//   4. completion: finished rays hand their result to the work item, which may start its next
//      ray in the same lane (e.g. the next sample of a pixel).
// Semantics are those of fast_trace(): the result is the lexicographic minimum (t, index) of the
// triangles passing the reference test below the incoming length.
#pragma once

#include "mrt_trace.cuh"

namespace mrt {

// the node phase of a warp ends when no lane searches any more, or when fewer than Q lanes search
// while others hold leaves: those leaves are tested first, and the few searching lanes go on in the
// next node phase.  Coherent camera rays do best with Q = 16 (the NoShadows trace of the
// 1,000,000-triangle soup frame: 1757 Mrays/s against 1757 at 20, 1715 at 24, 1575 at 32, 1610 at
// 8), the incoherent bounces of the wavefront with Q = 4 (terrain PathTracer: 3, 4 and 6 within
// 0.3 %, 8 1.5 % slower).
#ifndef MRT_NODE_QUORUM
#define MRT_NODE_QUORUM 4
#endif
constexpr int kNodeQuorum = MRT_NODE_QUORUM;
#ifndef MRT_CAMERA_QUORUM
#define MRT_CAMERA_QUORUM 16
#endif
constexpr int kCameraQuorum = MRT_CAMERA_QUORUM;   // for a pass of camera rays (the NoShadows trace)
template <int Q = kNodeQuorum>
__device__ __forceinline__ bool node_phase_over(bool searching, bool holding_leaf) {
    const uint32_t s = __ballot_sync(0xFFFFFFFFu, searching);
    return s == 0u || (__popc(s) < Q && __any_sync(0xFFFFFFFFu, holding_leaf));
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
__device__ __forceinline__ void start_ray(const DevScene &s, const Ray &r, FastTrav &t) {
    float len = kRayLengthMax;
    uint32_t id = MRT_HIT_NONE;
    naive_trace<kPlane>(s, r, len, id);
    naive_trace<kSphere>(s, r, len, id);
    trav_begin<kCount>(s, r, len, id, t);   // the plane or sphere hit stays the answer unless a triangle is closer
}

// idle lanes of a warp that trigger a refill (all idle lanes refill then, with one atomic)
#ifndef MRT_REFILL_MIN
#define MRT_REFILL_MIN 8
#endif
constexpr int kRefillMin = MRT_REFILL_MIN;

template <bool kCount, class Work, class Lane, class Stack, int Q = kNodeQuorum, int R = kRefillMin>
__device__ void persistent_closest(const DevScene &s, Work &work, Lane &lane, Stack &stk) {
    const uint32_t FULL = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const uint32_t total = work.total();
    bool active = false;
    bool exhausted = false;
    Ray r;
    FastTrav t;
    for (;;) {
        // 1. refill idle lanes (one atomic per warp)
        const uint32_t idle = __ballot_sync(FULL, !active);
        if (!exhausted && (__popc(idle) >= R || idle == FULL)) {
            const int leader = __ffs(idle) - 1;
            uint32_t base = 0;
            if (lane_id == leader) base = atomicAdd(work.counter(), (uint32_t)__popc(idle));
            base = __shfl_sync(FULL, base, leader);
            if (base + (uint32_t)__popc(idle) >= total) exhausted = true;
            if (!active) {
                const uint32_t item = base + __popc(idle & ((1u << lane_id) - 1u));
                if (item < total && work.begin(item, lane, r)) {
                    start_ray<kCount, Work, Lane>(work.scene(lane, s), r, t);
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
            if (node_phase_over<Q>(w, active && trav_has_leaf(t))) break;
            if (w || (active && trav_can_speculate(t))) trav_node_step<kCount>(work.view(lane, s), r, t, stk);
        }
        // 3. leaf phase
        if (active && trav_has_leaf(t)) trav_leaf_step<kCount>(work.view(lane, s), r, t);
        // 4. completion
        if (active && trav_finished(t)) {
            float len = t.best_t;
            uint32_t id = t.best_id;
            const bool hit_light = lights_trace(work.scene(lane, s), r, len, id);
            const bool hit = id != MRT_HIT_NONE || hit_light;
            if (work.finish(lane, r, hit, len, id, t)) start_ray<kCount, Work, Lane>(work.scene(lane, s), r, t);
            else active = false;
        }
    }
}

// the same with the stack in local memory
template <bool kCount, int Q = kNodeQuorum, int R = kRefillMin, class Work, class Lane>
__device__ __forceinline__ void persistent_closest(const DevScene &s, Work &work, Lane &lane) {
    TravStack stk;
    persistent_closest<kCount, Work, Lane, TravStack, Q, R>(s, work, lane, stk);
}

}  // namespace mrt

namespace mrt {

// ---------------------------------------------------------------------------------------------
// any-hit (Shader::shadowTrace, Shader.cpp:162-187): planes and spheres in order, then the tree;
// the first occluder ends the ray, so no ordering and no distance culling beyond `dist`.
// Work provides total(), counter(), scene(lane, s), begin(item, lane, r, dist) and finish(lane, occluded).
// ---------------------------------------------------------------------------------------------
// the any-hit query keeps the shadow distance in best_t; planes and spheres are tested in order
// first, then the tree, where the first occluding triangle ends the query
__device__ __forceinline__ void occ_begin(const DevScene &s, const Ray &r, float dist, FastTrav &t) {
    trav_begin<false>(s, r, dist, MRT_HIT_NONE, t);
    if (naive_occ<kPlane>(s, r, dist) || naive_occ<kSphere>(s, r, dist)) {
        trav_set_occluded(t);
        trav_clear(t);
    }
}

#ifndef MRT_SHADOW_QUORUM
#define MRT_SHADOW_QUORUM 4
#endif
// node-phase quorum of any-hit (shadow) rays (terrain PathTracer and glass room: 4, 8 and 16 within 0.3 %)
constexpr int kShadowQuorum = MRT_SHADOW_QUORUM;

template <class Work, class Lane>
__device__ void persistent_any(const DevScene &s, Work &work, Lane &lane) {
    const uint32_t FULL = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const uint32_t total = work.total();
    bool active = false;
    bool exhausted = false;
    Ray r;
    FastTrav t;
    TravStack stk;
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
            const bool w = active && trav_wants_node(t);
            if (node_phase_over<kShadowQuorum>(w, active && trav_has_leaf(t))) break;
            if (w || (active && trav_can_speculate(t))) trav_node_step<false>(work.view(lane, s), r, t, stk);
        }
        if (active && trav_has_leaf(t)) trav_occ_leaf_step(work.view(lane, s), r, t);
        if (active && trav_finished(t)) {
            work.finish(lane, trav_hit(t));
            active = false;
        }
    }
}

}  // namespace mrt
