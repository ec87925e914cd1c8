/*
 * orc.h - CPU restatement of MobileRT's render path (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py may load liborc.so, and only as the checker.  The product (mobileraytracer_b200) never
 * links or calls it.
 *
 * Every function restates a reference function with the same float operation order (compiled with
 * -ffp-contract=off); the .c file cites the reference file:line for each.  Where the reference is
 * not reproducible (std::mt19937 seeded from /dev/urandom, process-wide atomic sample counters,
 * shuffled block order) the restatement draws from the keyed stream described in mrt_cuda.h, the
 * same stream the CUDA path consumes.  Pinning: the shapes, boxes, accelerators, camera and the
 * deterministic shader configurations are checked against the reference's own compiled code
 * (oracle/_ref/liboracle_ref.so) and the reference unit-test vectors (tests/test_oracle_*.py).
 */
#ifndef MRT_ORACLE_ORC_H
#define MRT_ORACLE_ORC_H

#include <stdint.h>
#include "../include/mrt_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Accelerators of the restatement: the reference's three, plus EXACT, a checker-only structure
 * whose closest hit is by construction the Naive closest hit (lowest index among equal t). */
#define ORC_ACCEL_NAIVE MRT_ACCEL_NAIVE
#define ORC_ACCEL_GRID MRT_ACCEL_REGULAR_GRID
#define ORC_ACCEL_BVH MRT_ACCEL_BVH
#define ORC_ACCEL_EXACT 3

typedef struct OrcScene OrcScene;

OrcScene *orc_scene_create(const MrtSceneDesc *desc);
void orc_scene_destroy(OrcScene *s);
/* accel: ORC_ACCEL_*; grid_size 0 = reference rule; grid_index MRT_GRID_INDEX_* */
int orc_scene_build(OrcScene *s, int accel, int grid_size, int grid_index, const float *camera_position);
/* grid bounds including the camera box [camera_min, camera_max] (orc_camera_box) */
int orc_scene_build_box(OrcScene *s, int accel, int grid_size, int grid_index, const float *camera_min,
                        const float *camera_max);
void orc_camera_box(const MrtCamera *c, float *mn, float *mx);
int orc_scene_grid_size(const OrcScene *s, int type);
uint64_t orc_scene_bvh_nodes(const OrcScene *s, int type);

void orc_trace_closest(OrcScene *s, const MrtRay *rays, uint32_t n, MrtHit *hits, int threads);
void orc_trace_any(OrcScene *s, const MrtRay *rays, const float *dist, uint32_t n, uint8_t *occ, int threads);
/* per ray: cells visited and triangle references tested by the triangle grid (grid scenes only) */
int orc_grid_counts(OrcScene *s, const MrtRay *rays, uint32_t n, uint32_t *cells, uint32_t *refs, int threads);

/* Whole frame (Renderer::renderFrame restated) with the keyed stream. bitmap: row pitch
 * stride_bytes/4; accum: optional 4 floats per pixel (width*height), summed in sample order. */
int orc_render(OrcScene *s, const MrtCamera *cam, const MrtRenderOpts *o, uint32_t *bitmap,
               uint32_t stride_bytes, float *accum, uint64_t *ray_counts, int threads);
/* Per-sample fp32 values of a list of pixels (x, y pairs), spp samples each:
 * out[(k * spp + s) * 3 + c]. */
int orc_render_pixels(OrcScene *s, const MrtCamera *cam, const MrtRenderOpts *o, const uint32_t *xy,
                      uint32_t n, float *out, int threads);

/* ---- single functions, for known-answer tests ---- */
int orc_triangle_intersect(const float *abc, const float *normals, const float *colors, const float *o,
                           const float *d, float length, float *out_t, float *out_normal, float *out_color);
int orc_triangle_occludes(const float *abc, const float *o, const float *d, float dist);
int orc_triangle_intersect_box(const float *abc, const float *bmin, const float *bmax);
int orc_plane_intersect_box(const float *pn, const float *bmin, const float *bmax);
float orc_plane_distance(const float *pn, const float *q);
int orc_plane_intersect(const float *pn, const float *o, const float *d, float length, float *out_t);
int orc_sphere_intersect(const float *cr, const float *o, const float *d, float length, float *out_t, float *out_n);
int orc_sphere_intersect_box(const float *cr, const float *bmin, const float *bmax);
int orc_aabb_intersect(const float *bmin, const float *bmax, const float *o, const float *d);
/* raster preview of the scene triangles (MainRenderer.copyFrame); counts[0] = triangles drawn after
 * clipping, counts[1] = covered pixel samples; 0 on success */
int orc_raster_preview(const MrtSceneDesc *d, const MrtCamera *cam, uint32_t width, uint32_t height, uint32_t *bitmap,
                       uint32_t stride_bytes, uint64_t *counts);
float orc_aabb_area(const float *bmin, const float *bmax);
float orc_halton(uint32_t index, uint32_t base);
uint32_t orc_incremental_avg(const float *rgb, uint32_t avg, uint32_t n);
void orc_camera_ray(const MrtCamera *c, float u, float v, float du, float dv, float *o6);
float orc_sample(const MrtRenderOpts *o, int kind, uint32_t pixel, uint32_t sample, uint32_t node, uint32_t dim);
void orc_sincos(float x, float *s, float *c);

#ifdef __cplusplus
}
#endif

#endif
