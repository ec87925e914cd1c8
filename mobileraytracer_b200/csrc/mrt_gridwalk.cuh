// mrt_gridwalk.cuh - persistent closest-hit engine for the RegularGrid (RegularGrid.hpp:157-337).
//
// grid_trace() walks one ray from its first cell to its last in one thread, so a warp waits for
// its longest walk (a camera ray that leaves the grid after a few cells shares the warp with one
// that crosses the dense soup for a hundred).  Here every lane keeps a resumable walk: the DDA
// state, the phase of the reference's two-phase loop (the first walk until a primitive reports a
// hit, then `testloop`, which re-tests the whole current cell and keeps stepping while the hit lies
// beyond the next cell boundary), the running length and hit id, and its step count.  The warp loops:
//   1. refill: idle lanes take new work items from a global counter (one atomicAdd per warp);
//   2. one cell per active lane, in that lane's phase;
//   3. completion: the area lights (Scene::traceLights, after the accelerators) and the work item's
//      finish(), which may start the item's next ray in the same lane.
// Every ray takes exactly grid_trace's steps in grid_trace's order, so the answer is the
// reference's bit for bit; only the interleaving across rays changes.
#pragma once

#include "mrt_persistent.cuh"

namespace mrt {

struct GridWalk {
    Dda st;
    float len;
    uint32_t id;
    uint32_t steps;
    uint8_t phase;   // 1: first walk, 2: testloop, 0: finished
    bool tri_hit;    // a triangle of the grid accepted (ends the first walk)
};

// planes and spheres walk their own grids first (Shader.cpp:124-150), whole, in this lane
__device__ __forceinline__ void grid_walk_begin(const DevScene &s, const Ray &r, GridWalk &w) {
    w.len = kRayLengthMax;
    w.id = MRT_HIT_NONE;
    w.tri_hit = false;
    grid_trace<kPlane>(s, r, w.len, w.id);
    grid_trace<kSphere>(s, r, w.len, w.id);
    w.steps = 0;
    const DevGrid &g = s.grid[kTriangle];
    if (!g.has) { w.phase = 0; return; }
    dda_setup(g, r, w.st);
    w.phase = 1;
}

// one cell of the lane's walk (RegularGrid.hpp:236-335)
__device__ __forceinline__ void grid_walk_step(const DevScene &s, const Ray &r, GridWalk &w) {
    const DevGrid &g = s.grid[kTriangle];
    const uint32_t c = grid_cell(g, w.st.X, w.st.Y, w.st.Z);
    const uint32_t b = __ldg(&g.start[c]), e = __ldg(&g.start[c + 1]);
    if (w.phase == 1) {
        for (uint32_t k = b; k < e; ++k) {
            w.tri_hit |= triangle_hit(s, __ldg(&g.refs[k]), r, w.len, w.id);
            if (w.tri_hit) { w.phase = 2; return; }   // testloop starts over this same cell
        }
        if (!dda_step(w.st)) { w.phase = 0; return; }
        if (++w.steps > kMaxGridSteps) { raise_error(s, MRT_ERR_LIMIT); w.phase = 0; }
        return;
    }
    for (uint32_t k = b; k < e; ++k) triangle_hit(s, __ldg(&g.refs[k]), r, w.len, w.id);
    Dda &st = w.st;
    bool out;
    if (st.tx < st.ty) {
        if (st.tx < st.tz) {
            out = w.len < st.tx;
            if (!out) { st.X += st.sx; out = st.X == st.ox; if (!out) st.tx = st.tx + st.dx; }
        } else {
            out = w.len < st.tz;
            if (!out) { st.Z += st.sz; out = st.Z == st.oz; if (!out) st.tz = st.tz + st.dz; }
        }
    } else {
        if (st.ty < st.tz) {
            out = w.len < st.ty;
            if (!out) { st.Y += st.sy; out = st.Y == st.oy; if (!out) st.ty = st.ty + st.dy; }
        } else {
            out = w.len < st.tz;
            if (!out) { st.Z += st.sz; out = st.Z == st.oz; if (!out) st.tz = st.tz + st.dz; }
        }
    }
    if (out) { w.phase = 0; return; }
    if (++w.steps > kMaxGridSteps) { raise_error(s, MRT_ERR_LIMIT); w.phase = 0; }
}

// Work provides total(), counter(), begin(item, lane, r) and
// finish(lane, r, hit, t, id, const FastTrav &) -> true: r holds the item's next ray (as persistent_closest)
template <class Work, class Lane>
__device__ void persistent_grid_closest(const DevScene &s, Work &work, Lane &lane) {
    const uint32_t FULL = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const uint32_t total = work.total();
    bool active = false;
    bool exhausted = false;
    Ray r;
    GridWalk w;
    const FastTrav none{};
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
                if (item < total && work.begin(item, lane, r)) {
                    grid_walk_begin(s, r, w);
                    active = true;
                }
            }
        }
        if (__ballot_sync(FULL, active) == 0) {
            if (exhausted) break;
            continue;
        }
        if (active && w.phase != 0) grid_walk_step(s, r, w);
        if (active && w.phase == 0) {
            lights_trace(s, r, w.len, w.id);
            // an accepted plane, sphere, triangle or light leaves its id
            if (work.finish(lane, r, w.id != MRT_HIT_NONE, w.len, w.id, none)) grid_walk_begin(s, r, w);
            else active = false;
        }
    }
}

}  // namespace mrt
