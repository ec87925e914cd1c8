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

// resident blocks of 128 threads per SM for the kernels of the persistent grid walk (7: 72 registers,
// no spills; 285 Mrays/s on that frame against 270 at 8 and 247 at 6)
#ifndef MRT_GRID_BLOCKS_PER_SM
#define MRT_GRID_BLOCKS_PER_SM 7
#endif
constexpr int kGridBlocksPerSm = MRT_GRID_BLOCKS_PER_SM;

// A lane's walk advances by one reference test or one cell step per iteration, so the lanes of a warp do
// the same small piece of work each iteration (a whole cell per iteration: 207 against 285 Mrays/s on the
// 1080p soup frame at G = 128, before the packed triangle records).
struct GridWalk {
    Dda st;
    float len;
    uint32_t id;
    uint32_t steps;
    uint32_t b, k, e;   // the current cell's references: first, next to test, end
    uint8_t phase;      // 1: first walk, 2: testloop, 0: finished
    bool tri_hit;       // a triangle of the grid accepted (ends the first walk)
};

__device__ __forceinline__ void grid_walk_load(const DevGrid &g, GridWalk &w) {
    const uint32_t c = grid_cell(g, w.st.X, w.st.Y, w.st.Z);
    w.b = __ldg(&g.start[c]);
    w.e = __ldg(&g.start[c + 1]);
    w.k = w.b;
}

// triangle i of the grid with the reference accept rule (triangle_hit), its edges from the grid's
// packed record when the build made them
__device__ __forceinline__ bool grid_tri_hit(const DevScene &s, const DevGrid &g, uint32_t i, const Ray &r, float &len,
                                             uint32_t &id) {
    if (!g.trec) return triangle_hit(s, i, r, len, id);
    const uint32_t self = hid(MRT_PRIM_TRIANGLE, i);
    if (r.exclude == self) return false;
    const float *rec = g.trec + 16 * (size_t)i;
    uint4 p0, p1;
    ldg_32b(reinterpret_cast<const uint4 *>(rec), p0, p1);
    const float acz = __ldg(rec + 8);
    const V3 a{__uint_as_float(p0.x), __uint_as_float(p0.y), __uint_as_float(p0.z)};
    const V3 ab{__uint_as_float(p0.w), __uint_as_float(p1.x), __uint_as_float(p1.y)};
    const V3 ac{__uint_as_float(p1.z), __uint_as_float(p1.w), acz};
    float t, u, v;
    if (!tri_test(a, ab, ac, r, t, u, v)) return false;
    if (t >= len) return false;
    len = t;
    id = self;
    return true;
}

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
    grid_walk_load(g, w);
    w.phase = 1;
}

// the testloop's move to the next cell (RegularGrid.hpp:282-335): false when the hit lies before the
// next cell boundary or the walk leaves the grid
__device__ __forceinline__ bool grid_testloop_step(GridWalk &w) {
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
    return !out;
}

// one reference of the current cell, or the move to the next cell (RegularGrid.hpp:236-335)
__device__ __forceinline__ void grid_walk_step(const DevScene &s, const Ray &r, GridWalk &w) {
    const DevGrid &g = s.grid[kTriangle];
    if (w.k < w.e) {
        // (loading the next reference's index one test ahead was slower: 304 against 322 Mrays/s)
        const bool h = grid_tri_hit(s, g, __ldg(&g.refs[w.k]), r, w.len, w.id);
        ++w.k;
        if (w.phase == 1 && h) {   // the first walk ends; the testloop starts over this same cell
            w.tri_hit = true;
            w.phase = 2;
            w.k = w.b;
        }
        return;
    }
    const bool more = w.phase == 1 ? dda_step(w.st) : grid_testloop_step(w);
    if (!more) { w.phase = 0; return; }
    if (++w.steps > kMaxGridSteps) { raise_error(s, MRT_ERR_LIMIT); w.phase = 0; return; }
    grid_walk_load(g, w);
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
