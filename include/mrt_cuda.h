/*
 * mrt_cuda.h - C ABI of the B200 render path for MobileRT (MobileRayTracer).
 *
 * Plain C types only: pointers, sizes and POD structs.  Every entry point returns an MRT_* status
 * code; the text of the last failure on a context is available from mrt_context_error().  No call
 * falls back to the CPU: if the CUDA device or the kernels are unavailable the call fails.
 *
 * Which reference interface each entry point replaces (paths inside the MobileRayTracer checkout):
 *   mrt_scene_create      Scene{triangles_, spheres_, planes_, materials_, lights_} filled by the caller
 *                         (app/MobileRT/Scene.hpp:23-27, filled in app/Scenes/Scenes.cpp:7-314 or
 *                         app/Components/ObjectLoaders/OBJLoader.cpp:68-248)
 *   mrt_obj_load          OBJLoader::process + OBJLoader::fillScene
 *                         (app/Components/ObjectLoaders/OBJLoader.cpp:21-248)
 *   mrt_scene_build       Shader::initializeAccelerators(Camera*)   (app/MobileRT/Shader.cpp:31-122)
 *                         -> Naive<T>, RegularGrid<T>, BVH<T> constructors
 *   mrt_trace_closest     Shader::rayTrace's accelerator part: planes -> spheres -> triangles -> lights
 *                         (app/MobileRT/Shader.cpp:124-150; BVH<T>::trace BVH.hpp:158-213,
 *                         RegularGrid<T>::trace RegularGrid.hpp:157-337, Naive<T>::trace Naive.hpp:56-63)
 *   mrt_trace_any         Shader::shadowTrace(ray, dist)             (app/MobileRT/Shader.cpp:162-187)
 *   mrt_render            Renderer::renderFrame(bitmap, numThreads, stride)
 *                         (app/MobileRT/Renderer.cpp:31-59, renderScene :67-116) with the shader's
 *                         shade() (app/Components/Shaders/{NoShadows,Whitted,PathTracer}.cpp)
 *   mrt_render_stop       Renderer::stopRender()                     (app/MobileRT/Renderer.cpp:61-65)
 *   mrt_render_progress   Renderer::getSample()                      (app/MobileRT/Renderer.cpp:118-120)
 *   mrt_raster_preview    the Android front end's raster preview: MainRenderer.copyFrame +
 *                         copyFrameBuffer (app/src/main/java/puscas/mobilertapp/MainRenderer.java:
 *                         111-139, 338-546) over DrawView's initVerticesArray / initColorsArray /
 *                         initCameraArray (app/System_dependent/Android_JNI/DrawView.cpp:47-210) and
 *                         VertexShaderRaster.glsl / FragmentShaderRaster.glsl
 * mrt_render_noalloc, the mrt_batch_* and the mrt_serve_* calls have no counterpart in the reference
 * (the reference renders one frame per Renderer::renderFrame call).
 */
#ifndef MRT_CUDA_H
#define MRT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------- */
#define MRT_OK 0
#define MRT_ERR_ARG 1        /* invalid argument (null pointer, size out of range, bad enum) */
#define MRT_ERR_OOM 2        /* device allocation failed */
#define MRT_ERR_CUDA 3       /* a CUDA runtime call failed; the context may be unusable */
#define MRT_ERR_LIMIT 4      /* a traversal step cap or queue capacity was exceeded */
#define MRT_ERR_CANCELLED 5  /* mrt_render_stop() was called while a render was in flight */
#define MRT_ERR_STATE 6      /* call out of order (e.g. trace before mrt_scene_build) */

/* ---- enums (reference integer codes are kept where the reference has them) ----------------- */
/* Shader::Accelerator (app/MobileRT/Shader.hpp:34-38) */
#define MRT_ACCEL_NAIVE 0
#define MRT_ACCEL_REGULAR_GRID 1
#define MRT_ACCEL_BVH 2

/* BVH flavour.  REFERENCE rebuilds the reference tree (unsorted top-down SAH, leaf <= 2,
 * BVH.hpp:87-155,273-311) and walks it with the reference slab test in the reference order, so its
 * results equal BVH<T>::trace bit for bit, including the slab test's rejections.  FAST builds a
 * Morton-ordered tree on the device, compressed into 8-wide nodes with quantised boxes, and walks it
 * nearest child first with a conservative box test; its closest hit is the exact closest hit
 * (= Naive<T>), ties resolved to the lowest primitive index. */
#define MRT_BVH_FAST 0
#define MRT_BVH_REFERENCE 1

/* RegularGrid cell addressing.  The reference fills cells at x + y*G + z*G*G
 * (RegularGrid.hpp:134-138) but reads them at X + (Y << s) + (Z << 2s), s = bitCounter(G) - 1
 * (RegularGrid.hpp:237-241); both agree only for power-of-two G.  REFERENCE keeps that pair of
 * formulas (bit-exact with the reference at any G); LINEAR reads with the fill formula. */
#define MRT_GRID_INDEX_REFERENCE 0
#define MRT_GRID_INDEX_LINEAR 1

/* c_wrapper.cpp:444-486 shader codes: 1 Whitted, 2 PathTracer, 3 DepthMap, 4 DiffuseMaterial,
 * default NoShadows.  DEPTHMAP (DepthMap.cpp:19-26) shades a hit grey by its distance against
 * MrtRenderOpts.depth_point; DIFFUSE (DiffuseMaterial.cpp:16-38) by the first non-zero of the
 * material's Kd, Ks, Kt, Le (the primitive colour without material). */
#define MRT_SHADER_NOSHADOWS 0
#define MRT_SHADER_WHITTED 1
#define MRT_SHADER_PATHTRACER 2
#define MRT_SHADER_DEPTHMAP 3
#define MRT_SHADER_DIFFUSE 4

/* Samplers (app/Components/Samplers).  The reference draws from std::mt19937 seeded from
 * /dev/urandom and from process-wide atomic counters, so it is not reproducible; here every draw is
 * a pure function of (seed, pixel, sample, path node, dimension), identical on the GPU and in the
 * CPU oracle:
 *   CONSTANT    value (Constant.cpp:13-15)
 *   STRATIFIED  frac(sample / spp + r)                 (Stratified.cpp:14-23, counter -> sample)
 *   HALTON      frac(haltonSequence(sample, p_d) + r)  (HaltonSeq.cpp:14-22, Utils.cpp:36-45)
 *   RANDOM      hash                                    (MersenneTwister.cpp:9-15)
 * r is a per-(pixel, node, dimension) rotation from the same hash, p_d the d-th prime. */
#define MRT_SAMPLER_CONSTANT 0
#define MRT_SAMPLER_STRATIFIED 1
#define MRT_SAMPLER_HALTON 2
#define MRT_SAMPLER_RANDOM 3

#define MRT_LIGHT_POINT 0 /* Components::PointLight (PointLight.cpp:17-26) */
#define MRT_LIGHT_AREA 1  /* Components::AreaLight  (AreaLight.cpp:22-43)  */

#define MRT_CAMERA_PERSPECTIVE 0  /* Components::Perspective (Perspective.cpp:24-44) */
#define MRT_CAMERA_ORTHOGRAPHIC 1 /* Components::Orthographic (Orthographic.cpp:23-46) */

/* Hit ids: primitive type in the top two bits, index inside that type's array below. */
#define MRT_PRIM_PLANE 0u
#define MRT_PRIM_SPHERE 1u
#define MRT_PRIM_TRIANGLE 2u
#define MRT_PRIM_LIGHT 3u
#define MRT_HIT_ID(type, index) ((((uint32_t)(type)) << 30) | ((uint32_t)(index)))
#define MRT_HIT_TYPE(id) ((uint32_t)(id) >> 30)
#define MRT_HIT_INDEX(id) ((uint32_t)(id) & 0x3FFFFFFFu)
#define MRT_HIT_NONE 0xFFFFFFFFu

/* Buffer location flag for the trace/render entry points. */
#define MRT_MEM_HOST 0u   /* arguments are host pointers; the call copies in and out */
#define MRT_MEM_DEVICE 1u /* arguments are device pointers on the context's device */

/* ---- plain data types ---------------------------------------------------------------------- */
/* MobileRT::Material (app/MobileRT/Material.hpp:13-17) */
typedef struct MrtMaterial {
    float le[3];  /* emission */
    float kd[3];  /* diffuse reflection */
    float ks[3];  /* specular reflection */
    float kt[3];  /* specular transmission */
    float ior;    /* refractive index */
} MrtMaterial;

typedef struct MrtLightDesc {
    int32_t kind;       /* MRT_LIGHT_POINT or MRT_LIGHT_AREA */
    float p0[3];        /* point light: position; area light: triangle vertex A */
    float p1[3];        /* area light: vertex B */
    float p2[3];        /* area light: vertex C */
    MrtMaterial radiance;
} MrtLightDesc;

/* The Scene's vectors as flat host arrays (the CUDA side keeps its own device copies). */
typedef struct MrtSceneDesc {
    uint32_t n_triangles;
    const float *tri_abc;          /* 9 floats per triangle: A, B, C */
    const float *tri_normals;      /* 9 floats per triangle (nA, nB, nC) or NULL: all three =
                                      normalize(cross(C - A, B - A)) as in Triangle.cpp:10-17 */
    const float *tri_colors;       /* 9 floats per triangle or NULL (zero colours) */
    const int32_t *tri_material;   /* material index per triangle or NULL (-1 = use colours) */
    uint32_t n_spheres;
    const float *sphere_center_radius; /* 4 floats per sphere */
    const int32_t *sphere_material;
    uint32_t n_planes;
    const float *plane_point_normal;   /* 6 floats per plane (normal normalised by the library) */
    const int32_t *plane_material;
    uint32_t n_materials;
    const MrtMaterial *materials;
    uint32_t n_lights;
    const MrtLightDesc *lights;
} MrtSceneDesc;

typedef struct MrtAccelOpts {
    int32_t accelerator;       /* MRT_ACCEL_* */
    int32_t bvh_mode;          /* MRT_BVH_* */
    int32_t grid_size;         /* 0 = the reference rule (Shader.cpp:76-105); > 0 forces G for triangles */
    int32_t grid_index;        /* MRT_GRID_INDEX_* */
    float camera_position[3];  /* grid bounds include the camera (Shader.cpp:56-62) ... */
    const struct MrtCamera *camera;   /* ... or, when not NULL, this camera's getAABB (a point for
                                         Perspective, the film rectangle for Orthographic,
                                         Camera.cpp:39-44, Orthographic.cpp:36-46) */
} MrtAccelOpts;

/* MobileRT::Ray (app/MobileRT/Ray.hpp:14-17); exclude = hit id of the primitive the ray leaves
 * (the reference compares Ray::primitive_ pointers), MRT_HIT_NONE for camera rays. */
typedef struct MrtRay {
    float origin[3];
    float direction[3];
    int32_t depth;
    uint32_t exclude;
} MrtRay;

typedef struct MrtHit {
    float t;       /* Intersection::length_; 1e30 (RayLengthMax) on a miss */
    uint32_t id;   /* MRT_HIT_ID(type, index) or MRT_HIT_NONE */
} MrtHit;

typedef struct MrtCamera {
    int32_t kind;         /* MRT_CAMERA_PERSPECTIVE or MRT_CAMERA_ORTHOGRAPHIC */
    float position[3];
    float look_at[3];
    float up[3];
    float fov_h_deg;      /* Perspective(position, lookAt, up, hFov, vFov): degrees;       */
    float fov_v_deg;      /* Orthographic(position, lookAt, up, sizeH, sizeV): film size    */
} MrtCamera;

/* MrtRenderOpts.flags */
/* Whitted / PathTracer wavefront of a scene that mixes diffuse with mirror or glass materials: sort
 * each window of a level's rays by material class before shading them, so that a warp runs one
 * material branch.  Off by default: on a 1024x1024 glass room (16 spp) the sorted shading was 8 %
 * slower than shading the rays in queue order. */
#define MRT_RENDER_SHADE_QUEUES 1u

typedef struct MrtRenderOpts {
    int32_t shader;         /* MRT_SHADER_* */
    uint32_t width;         /* Renderer width_ / height_ */
    uint32_t height;
    uint32_t spp;           /* samples per pixel (Renderer samplesPixel_) */
    uint32_t spl;           /* samples per light (Shader samplesLight_) */
    int32_t pixel_sampler;  /* MRT_SAMPLER_* for the camera-ray jitter */
    float constant_value;   /* value of a CONSTANT sampler (the reference CLI uses 0.5) */
    int32_t light_sampler;  /* sampler of AreaLight::getPosition */
    int32_t rr_sampler;     /* PathTracer Russian-roulette sampler */
    int32_t depth_min;      /* RayDepthMin (reference 4): Russian roulette only beyond it */
    int32_t depth_max;      /* RayDepthMax (reference 8): shade() returns black beyond it */
    uint64_t seed;          /* stream key */
    uint32_t spp_offset;    /* index of the first sample: a progressive render continues the stream
                               and the running mean from here */
    uint32_t flags;         /* MRT_RENDER_* bits (0: the defaults) */
    float depth_point[3];   /* DepthMap maxPoint (DepthMap.cpp:14-17): depth = max(1 - t / (2 |p - o|), 0) */
    uint32_t reserved2;
} MrtRenderOpts;

typedef struct MrtRenderStats {
    uint64_t rays_closest;  /* closest-hit rays traced (camera + secondary) */
    uint64_t rays_shadow;   /* any-hit rays traced */
    uint64_t paths;         /* camera paths (pixel samples) */
    float device_ms;        /* device time of the render */
    float trace_ms;         /* of which the closest-hit traversal launches of a NoShadows / DepthMap /
                               DiffuseMaterial frame on the FAST BVH or the RegularGrid (the rest is
                               shading and the running mean); 0 for other renders */
    uint32_t kernel_launches;  /* kernels the render launched */
    uint32_t reserved;
} MrtRenderStats;

typedef struct MrtContext MrtContext;
typedef struct MrtScene MrtScene;
typedef struct MrtArena MrtArena;

/* ---- context -------------------------------------------------------------------------------- */
int mrt_context_create(int device, MrtContext **out);
void mrt_context_destroy(MrtContext *ctx);
const char *mrt_context_error(const MrtContext *ctx);
int mrt_context_synchronize(MrtContext *ctx);
/* Stream the context launches on (a cudaStream_t), for callers that order their own work. */
void *mrt_context_stream(MrtContext *ctx);

/* ---- device arena (no counterpart in the reference) ----------------------------------------- */
/* One device allocation of `bytes` from which contexts that use it carve every scene buffer
 * (geometry, trees, build scratch) and their render scratch: scenes come and go without cudaMalloc /
 * cudaFree, so building or evicting a scene never synchronises the device while other work runs, and
 * the sum of all resident scenes is bounded by the arena's size.  Several contexts on one device may
 * share an arena (e.g. one building scenes while another renders); it is thread-safe.  Freeing a
 * scene returns its blocks at once: destroy a scene only when no work that reads it is in flight. */
int mrt_arena_create(int device, uint64_t bytes, MrtArena **out);
/* MRT_ERR_STATE (and nothing freed) while buffers carved from the arena are alive. */
int mrt_arena_destroy(MrtArena *arena);
int mrt_arena_stats(MrtArena *arena, uint64_t *capacity, uint64_t *used, uint64_t *peak,
                    uint64_t *largest_free);
/* Later device allocations of ctx come from `arena` (NULL: cudaMalloc again); existing buffers keep
 * their origin. */
int mrt_context_set_arena(MrtContext *ctx, MrtArena *arena);

/* ---- scene ---------------------------------------------------------------------------------- */
int mrt_scene_create(MrtContext *ctx, const MrtSceneDesc *desc, MrtScene **out);
void mrt_scene_destroy(MrtScene *scene);
int mrt_scene_build(MrtScene *scene, const MrtAccelOpts *opts);
/* Hand a scene to another context on the same device (e.g. from a context that builds scenes on one
 * thread to the one that renders them); waits for the old context's work first.  No counterpart in
 * the reference. */
int mrt_scene_move(MrtScene *scene, MrtContext *ctx);
/* Device bytes held by the scene (geometry + accelerator), for footprint admission. */
uint64_t mrt_scene_device_bytes(const MrtScene *scene);
/* Accelerator statistics: nodes (reference BVH nodes, or 8-wide FAST nodes) or cells (grid),
 * references, grid size. */
int mrt_scene_accel_info(const MrtScene *scene, uint64_t *nodes, uint64_t *refs, int32_t *grid_size);

/* ---- scene files ---------------------------------------------------------------------------- */
/* OBJLoader::process + fillScene (app/Components/ObjectLoaders/OBJLoader.cpp:21-248): reads a
 * Wavefront OBJ and the MTL file the caller names (mtl_path may be NULL: no materials) and fills
 * *desc with the scene the reference loader would build: x negated, polygons split as fans, given
 * normals normalised (else the Triangle constructor's normal), vertex colours, Ks / 2,
 * Kt * (1 - d), emission scaled down to a largest component of 1, emitting faces as AreaLights,
 * equal materials merged.  *desc points into *out until mrt_obj_free(*out).  On failure returns
 * MRT_ERR_ARG with the reason in error[0 .. error_len). */
typedef struct MrtObjScene MrtObjScene;
int mrt_obj_load(const char *obj_path, const char *mtl_path, MrtObjScene **out, MrtSceneDesc *desc, char *error,
                 size_t error_len);
void mrt_obj_free(MrtObjScene *scene);

/* ---- traversal ------------------------------------------------------------------------------ */
int mrt_trace_closest(MrtScene *scene, const MrtRay *rays, uint32_t n, MrtHit *hits, uint32_t mem);
/* occluded[i] = 1 if any plane/sphere/triangle blocks rays[i] within (Epsilon, dist[i]) */
int mrt_trace_any(MrtScene *scene, const MrtRay *rays, const float *dist, uint32_t n,
                  uint8_t *occluded, uint32_t mem);
/* Counting replay of mrt_trace_closest: per ray, on the FAST BVH the 128-byte nodes and the
 * 48-byte triangle records fetched; on the regular grid the cells visited (node_fetch) and the
 * triangle references tested (tri_fetch).  Other accelerators return MRT_ERR_STATE. */
int mrt_trace_closest_counts(MrtScene *scene, const MrtRay *rays, uint32_t n, uint32_t *node_fetch,
                             uint32_t *tri_fetch, uint32_t mem);

/* ---- rendering ------------------------------------------------------------------------------ */
/* One Renderer::renderFrame: for sample = spp_offset .. spp_offset+spp-1 every pixel the reference's
 * 16x16 block schedule covers gets bitmap = incrementalAvg(rgb, bitmap, sample + 1); other pixels
 * are left untouched.  stride_bytes / 4 is the row pitch in pixels.  accum (optional, 4 floats per
 * pixel at width*height) receives the per-pixel sum of the fp32 sample values, in sample order.
 * With MRT_MEM_HOST the call returns once the result is in the caller's buffers; on the plain
 * rectangle (row pitch 4 * width) only the scheduled rows are copied, and page-locked buffers
 * (cudaHostAlloc / cudaHostRegister) let it copy finished rows out while it shades the rest. */
int mrt_render(MrtScene *scene, const MrtCamera *camera, const MrtRenderOpts *opts,
               uint32_t *bitmap, uint32_t stride_bytes, float *accum, uint32_t mem,
               MrtRenderStats *stats);
/* mrt_render without any device allocation (no counterpart in the reference).  For callers that
 * cannot allocate device memory while rendering: processes whose device memory belongs to another
 * allocator or to a fixed budget (an engine that hands the renderer a pool and forbids cudaMalloc),
 * and latency-critical threads that must not meet cudaMalloc / cudaFree's implicit device
 * synchronisation.  bitmap and accum are device pointers; all other scratch is one static device
 * array of 12 MiB at most that every GPU loading the library keeps until exit.  Supports the
 * plain-rectangle block schedule only (width a multiple of 16, stride_bytes = 4 * width,
 * height / (height / 16) == 16), samplesLight <= 4 and depth_max <= 10; anything larger returns
 * MRT_ERR_ARG.  The call returns when its work on the context's stream has finished.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  Calls share the array: calls that overlap on the GPU (two host threads, or two
 * contexts on one device) race.  mrt_render_stop and mrt_render_progress apply as for mrt_render. */
int mrt_render_noalloc(MrtScene *scene, const MrtCamera *camera, const MrtRenderOpts *opts, uint32_t *bitmap,
                       uint32_t stride_bytes, float *accum, MrtRenderStats *stats);
void mrt_render_stop(MrtScene *scene);
uint32_t mrt_render_progress(const MrtScene *scene);

/* ---- raster preview ---------------------------------------------------------------------------- */
/* The first image the Android front end shows: the scene's triangles drawn with one flat colour each
 * (the material's max(Kd, Ks, Kt, Le) per component, or the mean of the vertex colours for a
 * triangle without material), back faces culled, nearest surface kept (a later triangle wins a
 * depth tie), background 0.  The camera's position, direction and up give a look-at view with z
 * negated; Perspective cameras project with fovY = 0.918 x the vertical field of view, near 0.1,
 * far 1e38; Orthographic ones with the film half sizes.  Pixel (x, y) of the width x height frame
 * is written at bitmap row y from the top as R | G << 8 | B << 16 | A << 24 (the render bitmap's
 * format).  The reference draws with OpenGL ES, which is not available to this library: parity is
 * with the oracle's restatement of the same pipeline (no graphics driver has been run). */
typedef struct MrtRasterStats {
    uint64_t triangles;   /* scene triangles */
    uint64_t drawn;       /* front-facing triangles (after near/far clipping) that reached the rasteriser */
    uint64_t fragments;   /* pixel samples covered by them */
    float device_ms;      /* device time of the preview */
} MrtRasterStats;
int mrt_raster_preview(MrtScene *scene, const MrtCamera *camera, uint32_t width, uint32_t height,
                       uint32_t *bitmap, uint32_t stride_bytes, uint32_t mem, MrtRasterStats *stats);

/* ---- batched rendering (no counterpart in the reference) ------------------------------------ */
/* Many renders of different scenes, cameras, resolutions and spp as one stream of waves over a
 * common ray pool.  Each wave takes camera paths from the jobs that still have some (by the
 * batch's policy), traces them through all bounce levels and folds their values into each job's
 * bitmap; the wave's kernel sequence is captured once as a CUDA graph and replayed, and several
 * waves run at once on their own streams (the tail of one wave's bounce levels overlaps the bulk of
 * another's).  A job's bitmap and sums end bit for bit as mrt_render(..., MRT_MEM_DEVICE, ...) with
 * the same arguments would leave them (the per-pixel sample order is kept).  Jobs render scenes built with MRT_ACCEL_BVH + MRT_BVH_FAST on the batch's device, with the
 * plain-rectangle block schedule (width a multiple of 16, stride_bytes = 4 * width and
 * height / (height / 16) == 16); bitmap and accum are device pointers that stay valid, and scenes
 * stay alive, until the job is reported done. */
typedef struct MrtBatch MrtBatch;

typedef struct MrtBatchOpts {
    uint32_t wave_roots;     /* camera paths per wave; 0 = chosen by the autotuner */
    uint32_t block_threads;  /* threads per block of the traversal kernels: 64, 128 or 256; 0 = autotuner */
    uint32_t blocks_per_sm;  /* blocks per SM of the traversal kernels (1..16); 0 = autotuner */
    uint32_t max_jobs;       /* jobs outstanding at once (job table slots); 0 = 4096 */
    uint32_t max_depth;      /* largest depth_max of any job (sizes the ray pool); 0 = 8 */
    uint32_t max_spl;        /* largest samplesLight of any job (sizes the shadow queue); 0 = 4 */
    uint32_t no_graph;       /* 1: launch each wave's kernels one by one instead of a CUDA graph */
    uint32_t max_wave_roots; /* upper bound for the autotuner's wave size; 0 = 2^21 */
    uint32_t policy;         /* MRT_BATCH_SMALLEST_FIRST (0), MRT_BATCH_FIFO or MRT_BATCH_EQUAL_SHARE */
    uint32_t pipelines;      /* waves in flight at once (1..4), each with its own stream and ray pool;
                                0 = autotuner (buffers for 4 are allocated) */
    uint32_t kernel;         /* MRT_BATCH_KERNEL_WAVEFRONT (one launch per bounce level),
                                MRT_BATCH_KERNEL_PATHS (whole paths per lane, one launch), 0 = per
                                wave: whole paths when no job holds half of the wave */
} MrtBatchOpts;

#define MRT_BATCH_KERNEL_WAVEFRONT 1
#define MRT_BATCH_KERNEL_PATHS 2

/* Which jobs fill a wave: the fewest paths left first / submission order / an equal share each. */
#define MRT_BATCH_SMALLEST_FIRST 0
#define MRT_BATCH_FIFO 1
#define MRT_BATCH_EQUAL_SHARE 2

typedef struct MrtBatchJob {
    MrtScene *scene;
    MrtCamera camera;
    MrtRenderOpts opts;
    uint32_t *bitmap;        /* device pointer, 4-byte aligned: running mean as in mrt_render */
    uint32_t stride_bytes;
    float *accum;            /* device pointer (16-byte aligned) or NULL: per-pixel fp32 sums */
} MrtBatchJob;

typedef struct MrtBatchStats {
    uint64_t rays_closest;   /* closest-hit rays traced by completed and running waves */
    uint64_t rays_shadow;
    uint64_t paths;          /* camera paths of the waves launched */
    uint64_t waves;          /* waves launched */
    uint64_t jobs_submitted;
    uint64_t jobs_done;
    double busy_ms;          /* device time with waves in flight (completed waves) */
    uint32_t wave_roots;     /* the settings in use (after autotuning) */
    uint32_t block_threads;
    uint32_t blocks_per_sm;
    uint32_t autotuned;      /* candidates the autotuner timed (0: fixed settings) */
    uint32_t pipelines;
    uint32_t kernel;         /* MRT_BATCH_KERNEL_* chosen for waves dominated by one job */
    uint64_t waves_paths;    /* waves run as whole-path launches */
} MrtBatchStats;

int mrt_batch_create(MrtContext *ctx, const MrtBatchOpts *opts, MrtBatch **out);
/* Waits for the batch's work on the device, then frees it. */
void mrt_batch_destroy(MrtBatch *batch);
/* Queue a job; its paths join the next wave.  MRT_ERR_LIMIT when max_jobs are outstanding. */
int mrt_batch_submit(MrtBatch *batch, const MrtBatchJob *job, uint64_t *job_id);
/* Launch up to max_waves waves without waiting for them (at most 8 run ahead of the host);
 * *launched receives the count (0: no job has paths left). */
int mrt_batch_step(MrtBatch *batch, uint32_t max_waves, uint32_t *launched);
/* Ids of jobs that completed since the last call (their bitmap and sums are final). */
int mrt_batch_completed(MrtBatch *batch, uint64_t *ids, uint32_t capacity, uint32_t *count);
/* Step until every submitted job is done, then synchronize. */
int mrt_batch_run(MrtBatch *batch);
int mrt_batch_stats(const MrtBatch *batch, MrtBatchStats *stats);

/* ---- serving: render requests over time (no counterpart in the reference) -------------------------
 * Requests arrive while others render; each joins the batched renderer's next waves as soon as its
 * scene is resident.  Admission by device footprint: a scene is built (on the device, from the host
 * copy mrt_serve_add_scene made) when its estimated bytes (240 per triangle + 1 MiB, then the exact
 * size) plus its image fit budget_bytes, after evicting idle resident scenes least recently used
 * first; otherwise the request waits at the head of the queue.  A scene's image stays resident with
 * it (and on the host while the scene is evicted): a request with opts->spp_offset > 0 continues the
 * running mean (a progressive re-render), one with spp_offset 0 starts from a cleared image; requests
 * of one scene run one at a time in arrival order.  mrt_serve_poll admits, dispatches and launches
 * waves without waiting for them, and reports finished requests, whose image has been copied to the
 * host bitmap given at submit (width x height, row pitch 4 * width).  All calls come from one host
 * thread. */
typedef struct MrtServe MrtServe;
typedef struct MrtServeOpts {
    uint64_t budget_bytes;       /* device bytes for resident scenes and their images */
    uint64_t build_slack_bytes;  /* further arena bytes for the scratch of the scene being built */
    MrtBatchOpts batch;          /* the batched renderer behind the requests */
} MrtServeOpts;
typedef struct MrtServeStats {
    uint64_t submitted, completed, builds, evictions;
    uint64_t resident_bytes, peak_bytes;
    uint64_t rays_closest, rays_shadow;
} MrtServeStats;
int mrt_serve_create(int device, const MrtServeOpts *opts, MrtServe **out);
void mrt_serve_destroy(MrtServe *serve);
const char *mrt_serve_error(const MrtServe *serve);
/* copies the scene's arrays; accel says how its accelerator is built when it becomes resident */
int mrt_serve_add_scene(MrtServe *serve, const MrtSceneDesc *desc, const MrtAccelOpts *accel, uint64_t *scene_id);
int mrt_serve_submit(MrtServe *serve, uint64_t scene_id, const MrtCamera *camera, const MrtRenderOpts *opts,
                     uint32_t *bitmap, uint64_t *request_id);
/* up to capacity finished request ids in done[], their number in *count */
int mrt_serve_poll(MrtServe *serve, uint64_t *done, uint32_t capacity, uint32_t *count);
/* requests submitted and not yet reported by mrt_serve_poll */
int mrt_serve_pending(const MrtServe *serve, uint64_t *requests);
/* seconds from mrt_serve_submit to the poll that saw the request finish */
int mrt_serve_request_latency(const MrtServe *serve, uint64_t request_id, double *seconds);
int mrt_serve_stats(const MrtServe *serve, MrtServeStats *stats);

#ifdef __cplusplus
}
#endif

#endif /* MRT_CUDA_H */
