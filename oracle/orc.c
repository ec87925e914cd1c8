/*
 * orc.c - CPU restatement of MobileRT's render hot path (the oracle).  TEST INFRASTRUCTURE ONLY:
 * loaded by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker; the
 * product never calls it.  Build: oracle/Makefile (-O2 -ffp-contract=off, no fast-math).
 *
 * Every float expression keeps the operation order of the reference source it cites (paths inside
 * the MobileRayTracer checkout, app/...), and of oracle/shim/glm/glm.hpp for the GLM built-ins.
 * Random draws come from the keyed stream defined in include/mrt_cuda.h instead of std::mt19937.
 */
#include "orc.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#define EPS 1.0e-06f            /* Utils.hpp:37 Epsilon */
#define RAY_LENGTH_MAX 1.0e+30f /* Utils.hpp:33 RayLengthMax */
#define NUMBER_OF_BLOCKS 256u   /* Utils.hpp:36 */

/* ============================== parallel loop (pthreads) ====================================== */
typedef void (*par_body)(long i, void *ctx, uint64_t *counters);
typedef struct { long n, chunk; atomic_long next; par_body body; void *ctx; uint64_t counters[2]; pthread_mutex_t mu; } ParJob;
static void *par_worker(void *arg) {
    ParJob *j = (ParJob *)arg;
    uint64_t local[2] = {0, 0};
    for (;;) {
        const long b = atomic_fetch_add(&j->next, j->chunk);
        if (b >= j->n) break;
        const long e = b + j->chunk < j->n ? b + j->chunk : j->n;
        for (long i = b; i < e; ++i) j->body(i, j->ctx, local);
    }
    pthread_mutex_lock(&j->mu);
    j->counters[0] += local[0]; j->counters[1] += local[1];
    pthread_mutex_unlock(&j->mu);
    return NULL;
}
/* runs body(i) for i in [0, n) on `threads` threads; returns the summed per-thread counters */
static void par_for(long n, int threads, long chunk, par_body body, void *ctx, uint64_t *counters) {
    ParJob j;
    j.n = n; j.chunk = chunk > 0 ? chunk : 1; atomic_init(&j.next, 0); j.body = body; j.ctx = ctx;
    j.counters[0] = j.counters[1] = 0;
    pthread_mutex_init(&j.mu, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    int started = 0;
    for (int t = 1; t < threads; ++t) if (pthread_create(&tid[started], NULL, par_worker, &j) == 0) ++started;
    par_worker(&j);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    pthread_mutex_destroy(&j.mu);
    if (counters) { counters[0] = j.counters[0]; counters[1] = j.counters[1]; }
}

/* ============================== vector arithmetic (glm shim order) ============================ */
typedef struct { float x, y, z; } V3;
static inline V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline V3 vld(const float *p) { return v3(p[0], p[1], p[2]); }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 vscale(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vdivs(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline V3 vadds(V3 a, float s) { return v3(a.x + s, a.y + s, a.z + s); }
static inline V3 vsubs(V3 a, float s) { return v3(a.x - s, a.y - s, a.z - s); }
static inline float vdot(V3 a, V3 b) {
    const float px = a.x * b.x, py = a.y * b.y, pz = a.z * b.z;
    return (px + py) + pz;
}
static inline V3 vcross(V3 a, V3 b) {
    return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline float vlength(V3 v) { return sqrtf(vdot(v, v)); }
static inline V3 vnormalize(V3 v) { const float inv = 1.0f / sqrtf(vdot(v, v)); return vscale(v, inv); }
static inline float smin(float a, float b) { return (b < a) ? b : a; } /* std::min(a, b) */
static inline float smax(float a, float b) { return (a < b) ? b : a; } /* std::max(a, b) */
static inline V3 vmin(V3 a, V3 b) { return v3(smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)); }
static inline V3 vmax(V3 a, V3 b) { return v3(smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)); }
static inline int vany_pos(V3 a) { return a.x > 0.0f || a.y > 0.0f || a.z > 0.0f; }
static inline float vcomp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
static inline V3 vreflect(V3 i, V3 n) { const float d = vdot(n, i); return vsub(i, vscale(vscale(n, d), 2.0f)); }
static inline V3 vrefract(V3 i, V3 n, float eta) {
    const float d = vdot(n, i);
    const float k = 1.0f - (eta * eta) * (1.0f - d * d);
    if (k < 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const float s = eta * d + sqrtf(k);
    return vsub(v3(eta * i.x, eta * i.y, eta * i.z), v3(s * n.x, s * n.y, s * n.z));
}

/* ============================== primitives ==================================================== */
typedef struct { V3 mn, mx; } Box;

typedef struct {
    V3 ac, ab, a;       /* Triangle.hpp:16-18: AC_, AB_, pointA_ */
    V3 na, nb, nc;
    V3 ca, cb, cc;
    int32_t mat;
} Tri;
typedef struct { V3 center; float sq_radius; int32_t mat; } Sph;   /* Sphere.hpp:16-18 */
typedef struct { V3 normal, point; int32_t mat; } Pln;             /* Plane.hpp:188-190 */
typedef struct { V3 le, kd, ks, kt; float ior; } Mat;
typedef struct { int kind; V3 pos; Tri tri; Mat radiance; } Lgt;

typedef struct {
    V3 origin, dir;
    int32_t depth;
    uint32_t exclude;   /* Ray::primitive_ as a hit id */
} Ray;

typedef struct {
    V3 point, normal, color;   /* Intersection.hpp:15-21 */
    float length;
    int32_t mat;               /* materialId_ */
    int light;                 /* >= 0: material_ = &lights[light].radiance (AreaLight.cpp:37-43) */
    uint32_t prim;             /* primitive_ as a hit id (spheres: none, Sphere.cpp:48) */
    uint32_t id;               /* id of the primitive that produced this record */
} Isect;

static Tri tri_make(const float *p, const float *n, const float *c, int32_t mat) {
    /* Triangle.cpp:10-21 (computed normals), :23-38 (given normals and colours), :40-54 */
    Tri t;
    const V3 A = vld(p), B = vld(p + 3), C = vld(p + 6);
    t.ac = vsub(C, A);
    t.ab = vsub(B, A);
    t.a = A;
    if (n) {
        t.na = vld(n); t.nb = vld(n + 3); t.nc = vld(n + 6);
    } else {
        const V3 nn = vnormalize(vcross(t.ac, t.ab));
        t.na = nn; t.nb = nn; t.nc = nn;
    }
    if (c) { t.ca = vld(c); t.cb = vld(c + 3); t.cc = vld(c + 6); }
    else { t.ca = v3(0, 0, 0); t.cb = t.ca; t.cc = t.ca; }
    t.mat = mat;
    return t;
}

/* Triangle::intersect(Intersection*, Ray)  Triangle.cpp:57-103 */
static int tri_hit(const Tri *t, uint32_t self, const Ray *r, Isect *it) {
    if (r->exclude == self) return 0;
    const V3 perp = vcross(r->dir, t->ac);
    const float np = vdot(t->ab, perp);
    if (fabsf(np) < EPS) return 0;
    const float inv = 1.0f / np;
    const V3 vtc = vsub(r->origin, t->a);
    const float u = inv * vdot(vtc, perp);
    if (u < 0.0f || u > 1.0f) return 0;
    const V3 upp = vcross(vtc, t->ab);
    const float v = inv * vdot(r->dir, upp);
    if (v < 0.0f || (u + v) > 1.0f) return 0;
    const float dist = inv * vdot(t->ac, upp);
    if (dist < EPS || dist >= it->length) return 0;
    const float w = 1.0f - u - v;
    it->normal = vadd(vadd(vscale(t->na, w), vscale(t->nb, u)), vscale(t->nc, v));
    it->color = vadd(vadd(vscale(t->ca, w), vscale(t->cb, u)), vscale(t->cc, v));
    it->point = vadd(r->origin, vscale(r->dir, dist));
    it->length = dist;
    it->mat = t->mat;
    it->prim = self;
    it->id = self;
    it->light = -1;
    return 1;
}

/* Triangle::intersect(Ray, dist)  Triangle.cpp:105-136 */
static int tri_occ(const Tri *t, uint32_t self, const Ray *r, float dist) {
    if (r->exclude == self) return 0;
    const V3 perp = vcross(r->dir, t->ac);
    const float np = vdot(t->ab, perp);
    if (fabsf(np) < EPS) return 0;
    const float inv = 1.0f / np;
    const V3 vtc = vsub(r->origin, t->a);
    const float u = inv * vdot(vtc, perp);
    if (u < 0.0f || u > 1.0f) return 0;
    const V3 upp = vcross(vtc, t->ab);
    const float v = inv * vdot(r->dir, upp);
    if (v < 0.0f || (u + v) > 1.0f) return 0;
    const float d = inv * vdot(t->ac, upp);
    return d > EPS && d < dist;
}

/* Triangle::getAABB  Triangle.cpp:145-152 */
static Box tri_box(const Tri *t) {
    const V3 B = vadd(t->a, t->ab), C = vadd(t->a, t->ac);
    Box b;
    b.mn = vmin(t->a, vmin(B, C));
    b.mx = vmax(t->a, vmax(B, C));
    return b;
}

/* intersectRayAABB lambda of Triangle::intersectBox  Triangle.cpp:155-219.  The vector swap of
 * T_1/T_2 only ever matters for the component just written, so a per-axis swap is the same. */
static int edge_box(V3 orig, V3 vec, const Box *box) {
    float t_near = FLT_MIN, t_far = FLT_MAX;
    for (int k = 0; k < 3; ++k) {
        const float o = vcomp(orig, k), d = vcomp(vec, k);
        const float bmn = vcomp(box->mn, k), bmx = vcomp(box->mx, k);
        if (fabsf(d) < EPS) {
            if ((o < bmn) || ((o + d) > bmx)) return 0;
        } else {
            float t1 = (bmn - o) / d;
            float t2 = (bmx - o) / d;
            if (t1 > t2) { const float tmp = t1; t1 = t2; t2 = tmp; }
            t_near = smax(t1, t_near);
            t_far = smin(t2, t_far);
            if ((t_near > t_far) || (t_far < 0)) return 0;
        }
    }
    return 1;
}

/* Triangle::intersectBox  Triangle.cpp:154-246 */
static int tri_in_box(const Tri *t, const Box *box) {
    const V3 vec = vsub(box->mx, box->mn);
    const int iab = edge_box(t->a, t->ab, box);
    const int iac = edge_box(t->a, t->ac, box);
    const V3 B = vadd(t->a, t->ab), C = vadd(t->a, t->ac);
    const int ibc = edge_box(B, vsub(C, B), box);
    Ray r; r.origin = box->mn; r.dir = vec; r.depth = 1; r.exclude = MRT_HIT_NONE;
    Isect it; it.length = RAY_LENGTH_MAX;
    const int iray = tri_hit(t, 0u, &r, &it);
    const V3 perp = vcross(vec, t->ac);
    const int inside = fabsf(vdot(t->ab, perp)) < EPS;
    return iab || iac || ibc || iray || inside;
}

/* Sphere  Sphere.cpp:13-16 (ctor), :18-52, :54-83, :94-100, :102-123 */
static Sph sph_make(const float *cr, int32_t mat) {
    Sph s; s.center = vld(cr); s.sq_radius = cr[3] * cr[3]; s.mat = mat; return s;
}
static int sph_solve(const Sph *s, const Ray *r, float *t) {
    const V3 oc = vsub(s->center, r->origin);
    const float proj = vdot(oc, r->dir);
    const float ocm = vlength(oc);
    const float A = vdot(r->dir, r->dir);
    const float B = 2.0f * -proj;
    const float C = ocm * ocm - s->sq_radius;
    const float disc = B * B - 4.0f * A * C;
    if (disc < 0.0f) return 0;
    const float root = sqrtf(disc);
    const float d1 = -B + root, d2 = -B - root;
    *t = smin(d1, d2) / (2.0f * A);
    return 1;
}
static int sph_hit(const Sph *s, uint32_t self, const Ray *r, Isect *it) {
    float t;
    if (!sph_solve(s, r, &t)) return 0;
    if (t < 1.0e-05f || t >= it->length) return 0;
    it->point = vadd(r->origin, vscale(r->dir, t));
    it->normal = vnormalize(vsub(it->point, s->center));
    it->color = v3(1.0f, 1.0f, 1.0f);   /* Intersection.hpp:29 default primitiveColor */
    it->length = t;
    it->mat = s->mat;
    it->prim = MRT_HIT_NONE;
    it->id = self;
    it->light = -1;
    return 1;
}
static int sph_occ(const Sph *s, const Ray *r, float dist) {
    float t;
    if (!sph_solve(s, r, &t)) return 0;
    return t > 1.0e-05f && t < dist;
}
static Box sph_box(const Sph *s) {
    const float rad = sqrtf(s->sq_radius);
    Box b; b.mn = vsubs(s->center, rad); b.mx = vadds(s->center, rad); return b;
}
static int sph_in_box(const Sph *s, const Box *box) {
    float dmin = 0;
    for (int k = 0; k < 3; ++k) {
        const float c = vcomp(s->center, k), a = vcomp(box->mn, k), b = vcomp(box->mx, k);
        if (c < a) dmin = dmin + (c - a) * (c - a);
        else if (c > b) dmin = dmin + (c - b) * (c - b);
    }
    return dmin <= s->sq_radius;
}

/* Plane  Plane.cpp:11-15 (ctor), :17-45, :47-71, :80-97, :99-105, :107-124, :126-155 */
static Pln pln_make(const float *pn, int32_t mat) {
    Pln p; p.point = vld(pn); p.normal = vnormalize(vld(pn + 3)); p.mat = mat; return p;
}
static int pln_hit(const Pln *p, uint32_t self, const Ray *r, Isect *it) {
    if (r->exclude == self) return 0;
    const float np = vdot(p->normal, r->dir);
    if (fabsf(np) < EPS) return 0;
    const V3 vtp = vsub(p->point, r->origin);
    const float sp = vdot(p->normal, vtp);
    const float t = sp / np;
    if (t < EPS || t >= it->length) return 0;
    it->point = vadd(r->origin, vscale(r->dir, t));
    it->normal = p->normal;
    it->color = v3(1.0f, 1.0f, 1.0f);
    it->length = t;
    it->mat = p->mat;
    it->prim = self;
    it->id = self;
    it->light = -1;
    return 1;
}
static int pln_occ(const Pln *p, uint32_t self, const Ray *r, float dist) {
    if (r->exclude == self) return 0;
    const float np = vdot(p->normal, r->dir);
    if (fabsf(np) < EPS) return 0;
    const V3 vtp = vsub(p->point, r->origin);
    const float sp = vdot(p->normal, vtp);
    const float t = sp / np;
    return t > EPS && t < dist;
}
static Box pln_box(const Pln *p) {
    V3 right = v3(0, 0, 0);
    const V3 n = p->normal;
    if (n.x >= 1) right = v3(0, 1, 1);
    else if (n.y >= 1) right = v3(1, 0, 1);
    else if (n.z >= 1) right = v3(1, 1, 0);
    else if (n.x <= -1) right = v3(0, 1, 1);
    else if (n.y <= -1) right = v3(1, 0, 1);
    else if (n.z <= -1) right = v3(1, 1, 0);
    right = vnormalize(right);
    Box b;
    b.mn = vadd(p->point, vscale(right, -100.0f));
    b.mx = vadd(p->point, vscale(right, 100.0f));
    return b;
}
static float pln_distance(const Pln *p, V3 q) {
    const V3 n = p->normal, o = p->point;
    const float d = n.x * -o.x + n.y * -o.y + n.z * -o.z;
    const float num = n.x * q.x + n.y * q.y + n.z * q.z + d;
    const float den = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
    return num / den;
}
static int pln_in_box(const Pln *p, const Box *box) {
    const float dp = pln_distance(p, box->mx);
    const float dn = pln_distance(p, box->mn);
    return (dp <= 0 && dn >= 0) || (dp >= 0 && dn <= 0);
}

/* intersect(AABB, Ray)  AABB.cpp:15-35 */
static int box_hit(const Box *b, const Ray *r) {
    const float invx = 1.0f / r->dir.x;
    const float t1x = (b->mn.x - r->origin.x) * invx;
    const float t2x = (b->mx.x - r->origin.x) * invx;
    float tmin = smin(t1x, t2x);
    float tmax = smax(t1x, t2x);
    for (int k = 1; k < 3; ++k) {
        const float inv = 1.0f / vcomp(r->dir, k);
        const float o = vcomp(r->origin, k);
        const float t1 = (vcomp(b->mn, k) - o) * inv;
        const float t2 = (vcomp(b->mx, k) - o) * inv;
        tmin = smax(tmin, smin(t1, t2));
        tmax = smin(tmax, smax(t1, t2));
    }
    return tmax >= smax(tmin, 0.0f);
}
/* AABB::getSurfaceArea  AABB.cpp:37-49 */
static float box_area(const Box *b) {
    const float lx = b->mx.x - b->mn.x, ly = b->mx.y - b->mn.y, lz = b->mx.z - b->mn.z;
    const float bt = 2 * lx * lz, xy = 2 * lx * ly, zy = 2 * lz * ly;
    return bt + xy + zy;
}
/* surroundingBox(box1, box2)  AABB.cpp:52-60 */
static Box box_union(const Box *b1, const Box *b2) {
    Box r; r.mn = vmin(b1->mn, b2->mn); r.mx = vmax(b1->mx, b2->mx); return r;
}

/* ============================== type dispatch ================================================= */
enum { T_PLANE = 0, T_SPHERE = 1, T_TRI = 2 };

typedef struct {
    uint32_t n;
    int type;
    const void *prims;   /* Pln*, Sph* or Tri* */
} PrimSet;

static Box ps_box(const PrimSet *ps, uint32_t i) {
    switch (ps->type) {
        case T_PLANE: return pln_box((const Pln *)ps->prims + i);
        case T_SPHERE: return sph_box((const Sph *)ps->prims + i);
        default: return tri_box((const Tri *)ps->prims + i);
    }
}
static int ps_in_box(const PrimSet *ps, uint32_t i, const Box *b) {
    switch (ps->type) {
        case T_PLANE: return pln_in_box((const Pln *)ps->prims + i, b);
        case T_SPHERE: return sph_in_box((const Sph *)ps->prims + i, b);
        default: return tri_in_box((const Tri *)ps->prims + i, b);
    }
}
static int ps_hit(const PrimSet *ps, uint32_t i, const Ray *r, Isect *it) {
    switch (ps->type) {
        case T_PLANE: return pln_hit((const Pln *)ps->prims + i, MRT_HIT_ID(MRT_PRIM_PLANE, i), r, it);
        case T_SPHERE: return sph_hit((const Sph *)ps->prims + i, MRT_HIT_ID(MRT_PRIM_SPHERE, i), r, it);
        default: return tri_hit((const Tri *)ps->prims + i, MRT_HIT_ID(MRT_PRIM_TRIANGLE, i), r, it);
    }
}
static int ps_occ(const PrimSet *ps, uint32_t i, const Ray *r, float dist) {
    switch (ps->type) {
        case T_PLANE: return pln_occ((const Pln *)ps->prims + i, MRT_HIT_ID(MRT_PRIM_PLANE, i), r, dist);
        case T_SPHERE: return sph_occ((const Sph *)ps->prims + i, r, dist);
        default: return tri_occ((const Tri *)ps->prims + i, MRT_HIT_ID(MRT_PRIM_TRIANGLE, i), r, dist);
    }
}

/* ============================== BVH (reference tree)  BVH.hpp ================================= */
typedef struct { Box box; uint32_t offset, count; } BNode;
typedef struct { BNode *nodes; uint32_t n_nodes; } RefBvh;

/* getSplitIndex_SAH  BVH.hpp:273-311 (boxes of the node's primitives in input order) */
static uint32_t sah_split(const Box *boxes, uint32_t N, float *left_area, float *right_area) {
    const uint32_t L = 2; /* maxLeafSize, BVH.hpp:19 */
    Box lb = boxes[0];
    left_area[0] = box_area(&lb);
    for (uint32_t i = 1; i < N - L; ++i) { lb = box_union(&lb, &boxes[i]); left_area[i] = box_area(&lb); }
    for (uint32_t i = 0; i < N - L; ++i) right_area[i] = 0.0f;
    Box rb = boxes[N - 1];
    right_area[N - L - 1] = box_area(&rb);
    for (uint32_t i = N - 2; i > L; --i) { rb = box_union(&rb, &boxes[i]); right_area[i - L] = box_area(&rb); }
    uint32_t split = L;
    float min_sah = (float)L * left_area[L - 1] + (float)(N - L) * right_area[L - 1];
    for (uint32_t i = L; i < N - L; ++i) {
        const float sl = (float)(i + 1) * left_area[i];
        const float sr = (float)(N - (i + 1)) * right_area[i];
        const float sah = sl + sr;
        if (sah < min_sah) { split = i + 1; min_sah = sah; }
    }
    return split;
}

/* BVH<T>::BVH + build  BVH.hpp:64-75, 87-155 (node numbering reproduced) */
static void refbvh_build(RefBvh *bvh, const PrimSet *ps) {
    const uint32_t N = ps->n;
    if (N == 0) { bvh->nodes = calloc(1, sizeof(BNode)); bvh->n_nodes = 1; return; }
    BNode *nodes = calloc(2 * (size_t)N - 1, sizeof(BNode));
    Box *pboxes = malloc(sizeof(Box) * N);
    for (uint32_t i = 0; i < N; ++i) pboxes[i] = ps_box(ps, i);
    Box *boxes = malloc(sizeof(Box) * N);
    float *la = malloc(sizeof(float) * N), *ra = malloc(sizeof(float) * N);
    uint32_t st_id[512], st_b[512], st_e[512];
    memset(st_id, 0, sizeof(st_id)); memset(st_b, 0, sizeof(st_b)); memset(st_e, 0, sizeof(st_e));
    uint32_t sp = 1, id = 0, begin = 0, end = N, max_id = 0;
    do {
        BNode *nd = &nodes[id];
        nd->box = pboxes[begin];
        boxes[0] = nd->box;
        const uint32_t size = end - begin;
        for (uint32_t i = begin + 1; i < end; ++i) {
            nd->box = box_union(&pboxes[i], &nd->box);
            boxes[i - begin] = pboxes[i];
        }
        if (size <= 2) {
            nd->offset = begin; nd->count = size;
            --sp; id = st_id[sp]; begin = st_b[sp]; end = st_e[sp];
        } else {
            const uint32_t left = max_id + 1, right = left + 1;
            nd->offset = left;
            max_id = right > max_id ? right : max_id;
            const uint32_t split = size <= 4 ? 2 : sah_split(boxes, size, la, ra);
            st_id[sp] = right; st_b[sp] = begin + split; st_e[sp] = end; ++sp;
            id = left; end = begin + split;
        }
    } while (sp > 0);
    bvh->nodes = nodes;
    bvh->n_nodes = max_id + 1;
    free(pboxes); free(boxes); free(la); free(ra);
}

/* BVH<T>::trace  BVH.hpp:158-213 */
static int refbvh_trace(const RefBvh *bvh, const PrimSet *ps, const Ray *r, Isect *it) {
    if (ps->n == 0) return 0;
    uint32_t stack[512];
    uint32_t sp = 1, id = 0;
    stack[0] = 0;
    int hit = 0;
    do {
        const BNode *nd = &bvh->nodes[id];
        if (box_hit(&nd->box, r)) {
            if (nd->count > 0) {
                for (uint32_t i = 0; i < nd->count; ++i) hit |= ps_hit(ps, nd->offset + i, r, it);
                --sp; id = stack[sp];
            } else {
                const uint32_t left = nd->offset, right = left + 1;
                const int tl = box_hit(&bvh->nodes[left].box, r);
                const int tr = box_hit(&bvh->nodes[right].box, r);
                if (!tl && !tr) { --sp; id = stack[sp]; }
                else {
                    id = tl ? left : right;
                    if (tl && tr) { stack[sp] = right; ++sp; }
                }
            }
        } else { --sp; id = stack[sp]; }
    } while (sp > 0);
    return hit;
}

/* BVH<T>::shadowTrace  BVH.hpp:216-271 */
static int refbvh_occ(const RefBvh *bvh, const PrimSet *ps, const Ray *r, float dist) {
    if (ps->n == 0) return 0;
    uint32_t stack[512];
    uint32_t sp = 1, id = 0;
    stack[0] = 0;
    do {
        const BNode *nd = &bvh->nodes[id];
        if (box_hit(&nd->box, r)) {
            if (nd->count > 0) {
                for (uint32_t i = 0; i < nd->count; ++i) if (ps_occ(ps, nd->offset + i, r, dist)) return 1;
                --sp; id = stack[sp];
            } else {
                const uint32_t left = nd->offset, right = left + 1;
                const int tl = box_hit(&bvh->nodes[left].box, r);
                const int tr = box_hit(&bvh->nodes[right].box, r);
                if (!tl && !tr) { --sp; id = stack[sp]; }
                else {
                    id = tl ? left : right;
                    if (tl && tr) { stack[sp] = right; ++sp; }
                }
            }
        } else { --sp; id = stack[sp]; }
    } while (sp > 0);
    return 0;
}

/* ============================== RegularGrid  RegularGrid.hpp ================================== */
typedef struct {
    int32_t G;
    uint32_t shift;
    int index_mode;
    Box ext;
    V3 sr, cw;
    int has;
    uint32_t *start;   /* G^3 + 1 offsets into refs */
    uint32_t *refs;
} Grid;

static uint32_t bit_counter(uint32_t n) { uint32_t c = 0; while (n > 0) { ++c; n >>= 1; } return c; } /* Utils.cpp:26-33 */
static uint32_t round_up_pow2(uint32_t v) {   /* Utils.cpp:15-24 */
    --v; v |= v >> 1u; v |= v >> 2u; v |= v >> 4u; v |= v >> 8u; v |= v >> 16u; ++v; return v;
}
/* grid size rule  Shader.cpp:76-105 */
static int32_t grid_size_rule(uint32_t n) {
    const int32_t a = n > 6 ? (int32_t)round_up_pow2(bit_counter(n)) : 2;
    const int32_t b = (int32_t)(round_up_pow2(bit_counter((uint32_t)a)) / 2);
    const int32_t ab = a * b;
    return ab > a ? ab : a;
}

/* RegularGrid ctor + addPrimitives  RegularGrid.hpp:50-79, 88-154 */
static void grid_build(Grid *g, const PrimSet *ps, Box bounds, int32_t G, int index_mode) {
    g->G = G;
    g->shift = bit_counter((uint32_t)G) - 1;
    g->index_mode = index_mode;
    g->ext = bounds;
    const V3 size = vsub(bounds.mx, bounds.mn);
    g->sr = v3((float)G / size.x, (float)G / size.y, (float)G / size.z);
    g->cw = vscale(size, 1.0f / (float)G);
    g->has = ps->n > 0;
    const size_t ncell = (size_t)G * G * G;
    uint32_t *count = calloc(ncell + 1, sizeof(uint32_t));
    const float sx = bounds.mx.x - bounds.mn.x, sy = bounds.mx.y - bounds.mn.y, sz = bounds.mx.z - bounds.mn.z;
    const float dx = sx / G, dy = sy / G, dz = sz / G;
    const float rx = dx > 0 ? 1.0f / dx : 1.0f, ry = dy > 0 ? 1.0f / dy : 1.0f, rz = dz > 0 ? 1.0f / dz : 1.0f;
    /* two passes (count, then fill) over the same candidate cells in the same order */
    uint32_t *fill = NULL;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            g->start = malloc(sizeof(uint32_t) * (ncell + 1));
            uint32_t acc = 0;
            for (size_t c = 0; c < ncell; ++c) { g->start[c] = acc; acc += count[c]; }
            g->start[ncell] = acc;
            g->refs = malloc(sizeof(uint32_t) * (acc ? acc : 1));
            fill = calloc(ncell, sizeof(uint32_t));
        }
        for (uint32_t i = 0; i < ps->n; ++i) {
            const Box bd = ps_box(ps, i);
            int32_t x1 = (int32_t)((bd.mn.x - bounds.mn.x) * rx), x2 = (int32_t)((bd.mx.x - bounds.mn.x) * rx) + 1;
            x1 = x1 > 0 ? x1 : 0; x2 = (G - 1 < x2) ? G - 1 : x2; x2 = fabsf(sx) < EPS ? 0 : x2; x1 = (x2 < x1) ? x2 : x1;
            int32_t y1 = (int32_t)((bd.mn.y - bounds.mn.y) * ry), y2 = (int32_t)((bd.mx.y - bounds.mn.y) * ry) + 1;
            y1 = y1 > 0 ? y1 : 0; y2 = (G - 1 < y2) ? G - 1 : y2; y2 = fabsf(sy) < EPS ? 0 : y2; y1 = (y1 < y2) ? y1 : y2;
            int32_t z1 = (int32_t)((bd.mn.z - bounds.mn.z) * rz), z2 = (int32_t)((bd.mx.z - bounds.mn.z) * rz) + 1;
            z1 = z1 > 0 ? z1 : 0; z2 = (G - 1 < z2) ? G - 1 : z2; z2 = fabsf(sz) < EPS ? 0 : z2; z1 = (z1 < z2) ? z1 : z2;
            /* a NaN box gives negative cell indices (undefined behaviour in the reference): skipped */
            if (x1 < 0 || y1 < 0 || z1 < 0 || x2 < 0 || y2 < 0 || z2 < 0) continue;
            for (int32_t x = x1; x <= x2; ++x)
                for (int32_t y = y1; y <= y2; ++y)
                    for (int32_t z = z1; z <= z2; ++z) {
                        const size_t idx = (size_t)x + (size_t)y * (size_t)G + (size_t)z * (size_t)G * (size_t)G;
                        const V3 pos = v3(bounds.mn.x + x * dx, bounds.mn.y + y * dy, bounds.mn.z + z * dz);
                        Box cell; cell.mn = pos; cell.mx = vadd(pos, v3(dx, dy, dz));
                        if (ps_in_box(ps, i, &cell)) {
                            if (pass == 0) count[idx]++;
                            else g->refs[g->start[idx] + fill[idx]++] = i;
                        }
                    }
        }
    }
    free(count); free(fill);
}

static inline uint32_t grid_index(const Grid *g, int32_t X, int32_t Y, int32_t Z) {
    if (g->index_mode == MRT_GRID_INDEX_LINEAR)
        return (uint32_t)X + (uint32_t)Y * (uint32_t)g->G + (uint32_t)Z * (uint32_t)g->G * (uint32_t)g->G;
    return (uint32_t)X + ((uint32_t)Y << g->shift) + ((uint32_t)Z << (g->shift * 2u));
}

typedef struct { int32_t X, Y, Z, step[3], out[3]; float tmax[3], tdelta[3]; } Dda;

/* DDA setup shared by trace and shadowTrace  RegularGrid.hpp:161-231 */
static void dda_setup(const Grid *g, const Ray *r, Dda *s) {
    const V3 cell = vmul(vsub(r->origin, g->ext.mn), g->sr);
    int32_t c[3] = {(int32_t)cell.x, (int32_t)cell.y, (int32_t)cell.z};
    for (int k = 0; k < 3; ++k) { c[k] = c[k] > 0 ? c[k] : 0; c[k] = (g->G - 1 < c[k]) ? g->G - 1 : c[k]; }
    float cb[3];
    for (int k = 0; k < 3; ++k) {
        const float mn = vcomp(g->ext.mn, k), cw = vcomp(g->cw, k);
        if (vcomp(r->dir, k) > 0) { s->step[k] = 1; s->out[k] = g->G; cb[k] = mn + (c[k] + 1) * cw; }
        else { s->step[k] = -1; s->out[k] = -1; cb[k] = mn + c[k] * cw; }
    }
    for (int k = 0; k < 3; ++k) {
        s->tmax[k] = 0.0f; s->tdelta[k] = 0.0f;
        const float d = vcomp(r->dir, k);
        if (fabsf(d) > EPS) {
            const float rr = 1.0f / d;
            s->tmax[k] = (cb[k] - vcomp(r->origin, k)) * rr;
            s->tdelta[k] = vcomp(g->cw, k) * s->step[k] * rr;
        } else {
            s->tmax[k] = RAY_LENGTH_MAX;
        }
    }
    s->X = c[0]; s->Y = c[1]; s->Z = c[2];
}

/* one DDA step; returns 0 when the walk leaves the grid  RegularGrid.hpp:251-279 */
static int dda_step(Dda *s) {
    if (s->tmax[0] < s->tmax[1]) {
        if (s->tmax[0] < s->tmax[2]) {
            s->X += s->step[0]; if (s->X == s->out[0]) return 0; s->tmax[0] = s->tmax[0] + s->tdelta[0];
        } else {
            s->Z += s->step[2]; if (s->Z == s->out[2]) return 0; s->tmax[2] = s->tmax[2] + s->tdelta[2];
        }
    } else {
        if (s->tmax[1] < s->tmax[2]) {
            s->Y += s->step[1]; if (s->Y == s->out[1]) return 0; s->tmax[1] = s->tmax[1] + s->tdelta[1];
        } else {
            s->Z += s->step[2]; if (s->Z == s->out[2]) return 0; s->tmax[2] = s->tmax[2] + s->tdelta[2];
        }
    }
    return 1;
}

/* RegularGrid<T>::trace  RegularGrid.hpp:157-337 */
/* counts (optional): cells visited, references tested */
static int grid_trace_n(const Grid *g, const PrimSet *ps, const Ray *r, Isect *it, uint32_t *cells, uint32_t *refs) {
    if (!g->has) return 0;
    Dda s;
    dda_setup(g, r, &s);
    int hit = 0;
    for (;;) {
        const uint32_t idx = grid_index(g, s.X, s.Y, s.Z);
        int found = 0;
        if (cells) ++*cells;
        for (uint32_t k = g->start[idx]; k < g->start[idx + 1]; ++k) {
            if (refs) ++*refs;
            hit |= ps_hit(ps, g->refs[k], r, it);
            if (hit) { found = 1; break; }
        }
        if (found) break;
        if (!dda_step(&s)) return hit;
    }
    for (;;) {   /* testloop  RegularGrid.hpp:282-335 */
        const uint32_t idx = grid_index(g, s.X, s.Y, s.Z);
        if (cells) ++*cells;
        if (refs) *refs += g->start[idx + 1] - g->start[idx];
        for (uint32_t k = g->start[idx]; k < g->start[idx + 1]; ++k) hit |= ps_hit(ps, g->refs[k], r, it);
        if (s.tmax[0] < s.tmax[1]) {
            if (s.tmax[0] < s.tmax[2]) {
                if (it->length < s.tmax[0]) break;
                s.X += s.step[0]; if (s.X == s.out[0]) break; s.tmax[0] = s.tmax[0] + s.tdelta[0];
            } else {
                if (it->length < s.tmax[2]) break;
                s.Z += s.step[2]; if (s.Z == s.out[2]) break; s.tmax[2] = s.tmax[2] + s.tdelta[2];
            }
        } else {
            if (s.tmax[1] < s.tmax[2]) {
                if (it->length < s.tmax[1]) break;
                s.Y += s.step[1]; if (s.Y == s.out[1]) break; s.tmax[1] = s.tmax[1] + s.tdelta[1];
            } else {
                if (it->length < s.tmax[2]) break;
                s.Z += s.step[2]; if (s.Z == s.out[2]) break; s.tmax[2] = s.tmax[2] + s.tdelta[2];
            }
        }
    }
    return hit;
}

static int grid_trace(const Grid *g, const PrimSet *ps, const Ray *r, Isect *it) {
    return grid_trace_n(g, ps, r, it, NULL, NULL);
}

/* RegularGrid<T>::shadowTrace  RegularGrid.hpp:340-465 */
static int grid_occ(const Grid *g, const PrimSet *ps, const Ray *r, float dist) {
    if (!g->has) return 0;
    Dda s;
    dda_setup(g, r, &s);
    for (;;) {
        const uint32_t idx = grid_index(g, s.X, s.Y, s.Z);
        for (uint32_t k = g->start[idx]; k < g->start[idx + 1]; ++k)
            if (ps_occ(ps, g->refs[k], r, dist)) return 1;
        if (!dda_step(&s)) return 0;
    }
}

/* ============================== EXACT: checker-only Naive-equivalent BVH ====================== */
/* Median-split tree over primitive centroids with boxes padded outward and a double-precision
 * slab test that never rejects a box holding an accepted hit; leaves are tested with the reference
 * primitive test and the result is the lexicographic minimum (t, index) = the Naive<T> result. */
typedef struct { double mn[3], mx[3]; uint32_t left, right, first, count; } XNode;
typedef struct { XNode *nodes; uint32_t n_nodes; uint32_t *order; } XBvh;

static void xbvh_build(XBvh *x, const PrimSet *ps) {
    const uint32_t N = ps->n;
    x->order = malloc(sizeof(uint32_t) * (N ? N : 1));
    x->nodes = malloc(sizeof(XNode) * (2 * (size_t)(N ? N : 1)));
    x->n_nodes = 0;
    if (N == 0) return;
    double (*cent)[3] = malloc(sizeof(double) * 3 * N);
    double (*bmn)[3] = malloc(sizeof(double) * 3 * N), (*bmx)[3] = malloc(sizeof(double) * 3 * N);
    for (uint32_t i = 0; i < N; ++i) {
        const Box b = ps_box(ps, i);
        x->order[i] = i;
        for (int k = 0; k < 3; ++k) {
            const double lo = vcomp(b.mn, k), hi = vcomp(b.mx, k);
            const double pad = 1e-4 * (fabs(lo) + fabs(hi) + (hi - lo)) + 1e-30;
            bmn[i][k] = lo - pad; bmx[i][k] = hi + pad;
            cent[i][k] = 0.5 * (lo + hi);
        }
    }
    uint32_t stack[128][3];
    int sp = 0;
    x->nodes[0].first = 0; x->nodes[0].count = N;
    x->n_nodes = 1;
    stack[sp][0] = 0; stack[sp][1] = 0; stack[sp][2] = N; ++sp;
    while (sp > 0) {
        --sp;
        const uint32_t ni = stack[sp][0], b = stack[sp][1], e = stack[sp][2];
        XNode *nd = &x->nodes[ni];
        double cmn[3] = {1e300, 1e300, 1e300}, cmx[3] = {-1e300, -1e300, -1e300};
        for (int k = 0; k < 3; ++k) { nd->mn[k] = 1e300; nd->mx[k] = -1e300; }
        for (uint32_t j = b; j < e; ++j) {
            const uint32_t p = x->order[j];
            for (int k = 0; k < 3; ++k) {
                if (bmn[p][k] < nd->mn[k]) nd->mn[k] = bmn[p][k];
                if (bmx[p][k] > nd->mx[k]) nd->mx[k] = bmx[p][k];
                if (cent[p][k] < cmn[k]) cmn[k] = cent[p][k];
                if (cent[p][k] > cmx[k]) cmx[k] = cent[p][k];
            }
        }
        nd->first = b; nd->count = e - b; nd->left = nd->right = 0;
        if (e - b <= 4 || sp >= 126) continue;
        int ax = 0;
        for (int k = 1; k < 3; ++k) if (cmx[k] - cmn[k] > cmx[ax] - cmn[ax]) ax = k;
        if (!(cmx[ax] > cmn[ax])) continue;
        const double mid = 0.5 * (cmn[ax] + cmx[ax]);
        uint32_t i = b, j = e;
        while (i < j) {
            if (cent[x->order[i]][ax] < mid) ++i;
            else { --j; const uint32_t t = x->order[i]; x->order[i] = x->order[j]; x->order[j] = t; }
        }
        if (i == b || i == e) i = b + (e - b) / 2;
        const uint32_t l = x->n_nodes++, r = x->n_nodes++;
        nd->left = l; nd->right = r; nd->count = 0;
        stack[sp][0] = l; stack[sp][1] = b; stack[sp][2] = i; ++sp;
        stack[sp][0] = r; stack[sp][1] = i; stack[sp][2] = e; ++sp;
    }
    free(cent); free(bmn); free(bmx);
}

static int xbox_enter(const XNode *nd, const Ray *r, double tlimit) {
    double t0 = 0.0, t1 = tlimit;
    const double o[3] = {r->origin.x, r->origin.y, r->origin.z}, d[3] = {r->dir.x, r->dir.y, r->dir.z};
    for (int k = 0; k < 3; ++k) {
        if (d[k] == 0.0) {
            if (o[k] < nd->mn[k] || o[k] > nd->mx[k]) return 0;
            continue;
        }
        double a = (nd->mn[k] - o[k]) / d[k], b = (nd->mx[k] - o[k]) / d[k];
        if (a > b) { const double t = a; a = b; b = t; }
        if (a > t0) t0 = a;
        if (b < t1) t1 = b;
        if (t0 > t1) return 0;
    }
    return 1;
}

/* closest triangle among those accepted against length l0; returns 1 and fills it on success */
static int xbvh_trace(const XBvh *x, const PrimSet *ps, const Ray *r, Isect *it) {
    if (ps->n == 0 || x->n_nodes == 0) return 0;
    const float l0 = it->length;
    int have = 0;
    uint32_t best_i = 0;
    float best_t = l0;
    uint32_t stack[256];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const XNode *nd = &x->nodes[stack[--sp]];
        const double lim = have ? (double)best_t * (1.0 + 1e-5) + 1e-30 : (l0 >= RAY_LENGTH_MAX ? 1e300 : (double)l0 * (1.0 + 1e-5) + 1e-30);
        if (!xbox_enter(nd, r, lim)) continue;
        if (nd->count > 0) {
            for (uint32_t j = nd->first; j < nd->first + nd->count; ++j) {
                const uint32_t p = x->order[j];
                Isect tmp; tmp.length = RAY_LENGTH_MAX;
                if (!ps_hit(ps, p, r, &tmp)) continue;
                const float t = tmp.length;
                const int better = have ? (t < best_t || (t == best_t && p < best_i)) : (t < l0);
                if (better) { have = 1; best_t = t; best_i = p; }
            }
        } else {
            stack[sp++] = nd->right;
            stack[sp++] = nd->left;
        }
    }
    if (!have) return 0;
    Isect tmp; tmp.length = RAY_LENGTH_MAX;
    ps_hit(ps, best_i, r, &tmp);
    *it = tmp;
    return 1;
}

static int xbvh_occ(const XBvh *x, const PrimSet *ps, const Ray *r, float dist) {
    if (ps->n == 0 || x->n_nodes == 0) return 0;
    uint32_t stack[256];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const XNode *nd = &x->nodes[stack[--sp]];
        if (!xbox_enter(nd, r, (double)dist * (1.0 + 1e-5) + 1e-30)) continue;
        if (nd->count > 0) {
            for (uint32_t j = nd->first; j < nd->first + nd->count; ++j)
                if (ps_occ(ps, x->order[j], r, dist)) return 1;
        } else {
            stack[sp++] = nd->right;
            stack[sp++] = nd->left;
        }
    }
    return 0;
}

/* ============================== scene ========================================================= */
struct OrcScene {
    uint32_t n_tri, n_sph, n_pln, n_mat, n_light;
    Tri *tri; Sph *sph; Pln *pln; Mat *mat; Lgt *light;
    PrimSet sets[3];    /* planes, spheres, triangles */
    int accel;
    RefBvh bvh[3];
    Grid grid[3];
    XBvh xbvh[3];
    int built;
};

static Mat mat_load(const MrtMaterial *m) {
    Mat r; r.le = vld(m->le); r.kd = vld(m->kd); r.ks = vld(m->ks); r.kt = vld(m->kt); r.ior = m->ior; return r;
}

OrcScene *orc_scene_create(const MrtSceneDesc *d) {
    OrcScene *s = calloc(1, sizeof(OrcScene));
    s->n_tri = d->n_triangles; s->n_sph = d->n_spheres; s->n_pln = d->n_planes;
    s->n_mat = d->n_materials; s->n_light = d->n_lights;
    s->tri = malloc(sizeof(Tri) * (s->n_tri ? s->n_tri : 1));
    for (uint32_t i = 0; i < s->n_tri; ++i)
        s->tri[i] = tri_make(d->tri_abc + 9 * (size_t)i, d->tri_normals ? d->tri_normals + 9 * (size_t)i : NULL,
                             d->tri_colors ? d->tri_colors + 9 * (size_t)i : NULL, d->tri_material ? d->tri_material[i] : -1);
    s->sph = malloc(sizeof(Sph) * (s->n_sph ? s->n_sph : 1));
    for (uint32_t i = 0; i < s->n_sph; ++i)
        s->sph[i] = sph_make(d->sphere_center_radius + 4 * i, d->sphere_material ? d->sphere_material[i] : -1);
    s->pln = malloc(sizeof(Pln) * (s->n_pln ? s->n_pln : 1));
    for (uint32_t i = 0; i < s->n_pln; ++i)
        s->pln[i] = pln_make(d->plane_point_normal + 6 * i, d->plane_material ? d->plane_material[i] : -1);
    s->mat = malloc(sizeof(Mat) * (s->n_mat ? s->n_mat : 1));
    for (uint32_t i = 0; i < s->n_mat; ++i) s->mat[i] = mat_load(&d->materials[i]);
    s->light = malloc(sizeof(Lgt) * (s->n_light ? s->n_light : 1));
    for (uint32_t i = 0; i < s->n_light; ++i) {
        const MrtLightDesc *l = &d->lights[i];
        Lgt *g = &s->light[i];
        g->kind = l->kind;
        g->pos = vld(l->p0);
        float abc[9];
        memcpy(abc, l->p0, 12); memcpy(abc + 3, l->p1, 12); memcpy(abc + 6, l->p2, 12);
        g->tri = tri_make(abc, NULL, NULL, -1);   /* AreaLight.cpp:13-19: Triangle{A, B, C, -1} */
        g->radiance = mat_load(&l->radiance);
    }
    s->sets[T_PLANE].n = s->n_pln; s->sets[T_PLANE].type = T_PLANE; s->sets[T_PLANE].prims = s->pln;
    s->sets[T_SPHERE].n = s->n_sph; s->sets[T_SPHERE].type = T_SPHERE; s->sets[T_SPHERE].prims = s->sph;
    s->sets[T_TRI].n = s->n_tri; s->sets[T_TRI].type = T_TRI; s->sets[T_TRI].prims = s->tri;
    return s;
}

static void scene_free_accel(OrcScene *s) {
    for (int k = 0; k < 3; ++k) {
        free(s->bvh[k].nodes); s->bvh[k].nodes = NULL;
        free(s->grid[k].start); free(s->grid[k].refs); s->grid[k].start = NULL; s->grid[k].refs = NULL;
        free(s->xbvh[k].nodes); free(s->xbvh[k].order); s->xbvh[k].nodes = NULL; s->xbvh[k].order = NULL;
    }
    s->built = 0;
}

void orc_scene_destroy(OrcScene *s) {
    if (!s) return;
    scene_free_accel(s);
    free(s->tri); free(s->sph); free(s->pln); free(s->mat); free(s->light);
    free(s);
}

/* Shader::initializeAccelerators  Shader.cpp:31-122 */
int orc_scene_build(OrcScene *s, int accel, int grid_size, int grid_index_mode, const float *cam) {
    return orc_scene_build_box(s, accel, grid_size, grid_index_mode, cam, cam);
}

int orc_scene_build_box(OrcScene *s, int accel, int grid_size, int grid_index_mode, const float *cam_min,
                        const float *cam_max) {
    scene_free_accel(s);
    s->accel = accel;
    for (int k = 0; k < 3; ++k) {
        const PrimSet *ps = &s->sets[k];
        if (accel == ORC_ACCEL_BVH) refbvh_build(&s->bvh[k], ps);
        else if (accel == ORC_ACCEL_EXACT) xbvh_build(&s->xbvh[k], ps);
        else if (accel == ORC_ACCEL_GRID) {
            V3 mn = v3(RAY_LENGTH_MAX, RAY_LENGTH_MAX, RAY_LENGTH_MAX), mx = v3(-RAY_LENGTH_MAX, -RAY_LENGTH_MAX, -RAY_LENGTH_MAX);
            for (uint32_t i = 0; i < ps->n; ++i) {   /* Scene::getBounds / AABBbounds  Scene.cpp:42-45 */
                const Box b = ps_box(ps, i);
                mn = vmin(b.mn, mn);
                mx = vmax(b.mx, mx);
            }
            mn = vmin(vld(cam_min), mn);   /* the camera's getAABB (AABBbounds, Scene.cpp:42-45) */
            mx = vmax(vld(cam_max), mx);
            Box bounds; bounds.mn = vsubs(mn, EPS); bounds.mx = vadds(mx, EPS);
            int32_t G = grid_size_rule(ps->n);
            if (k == T_TRI && grid_size > 0) G = grid_size;
            grid_build(&s->grid[k], ps, bounds, G, grid_index_mode);
        }
    }
    s->built = 1;
    return 0;
}

int orc_scene_grid_size(const OrcScene *s, int type) { return s->grid[type].G; }
uint64_t orc_scene_bvh_nodes(const OrcScene *s, int type) { return s->bvh[type].n_nodes; }

static int accel_trace(const OrcScene *s, int k, const Ray *r, Isect *it) {
    const PrimSet *ps = &s->sets[k];
    switch (s->accel) {
        case ORC_ACCEL_BVH: return refbvh_trace(&s->bvh[k], ps, r, it);
        case ORC_ACCEL_GRID: return grid_trace(&s->grid[k], ps, r, it);
        case ORC_ACCEL_EXACT:
            if (k == T_TRI) return xbvh_trace(&s->xbvh[k], ps, r, it);
            /* planes and spheres are walked in order */
            /* fall through */
        default: {
            int hit = 0;
            for (uint32_t i = 0; i < ps->n; ++i) hit |= ps_hit(ps, i, r, it);   /* Naive.hpp:56-63 */
            return hit;
        }
    }
}

static int accel_occ(const OrcScene *s, int k, const Ray *r, float dist) {
    const PrimSet *ps = &s->sets[k];
    switch (s->accel) {
        case ORC_ACCEL_BVH: return refbvh_occ(&s->bvh[k], ps, r, dist);
        case ORC_ACCEL_GRID: return grid_occ(&s->grid[k], ps, r, dist);
        case ORC_ACCEL_EXACT:
            if (k == T_TRI) return xbvh_occ(&s->xbvh[k], ps, r, dist);
            /* fall through */
        default:
            for (uint32_t i = 0; i < ps->n; ++i) if (ps_occ(ps, i, r, dist)) return 1;   /* Naive.hpp:65-74 */
            return 0;
    }
}

/* Shader::rayTrace accelerator part + Scene::traceLights  Shader.cpp:124-150, Scene.cpp:31-37 */
static int scene_closest(const OrcScene *s, const Ray *r, Isect *it) {
    it->length = RAY_LENGTH_MAX;
    it->id = MRT_HIT_NONE;
    it->light = -1;
    it->mat = 0;
    int hit = 0;
    hit |= accel_trace(s, T_PLANE, r, it);
    hit |= accel_trace(s, T_SPHERE, r, it);
    hit |= accel_trace(s, T_TRI, r, it);
    for (uint32_t k = 0; k < s->n_light; ++k) {
        if (s->light[k].kind != MRT_LIGHT_AREA) continue;   /* PointLight::intersect is false */
        if (tri_hit(&s->light[k].tri, MRT_HIT_ID(MRT_PRIM_LIGHT, k), r, it)) {
            it->light = (int)k;
            hit = 1;
        }
    }
    return hit;
}

/* Shader::shadowTrace  Shader.cpp:162-187 */
static int scene_occ(const OrcScene *s, const Ray *r, float dist) {
    int occ = 0;
    occ |= accel_occ(s, T_PLANE, r, dist);
    occ |= accel_occ(s, T_SPHERE, r, dist);
    occ |= accel_occ(s, T_TRI, r, dist);
    return occ;
}

static Ray ray_from(const MrtRay *m) {
    Ray r; r.origin = vld(m->origin); r.dir = vld(m->direction); r.depth = m->depth; r.exclude = m->exclude; return r;
}

typedef struct { OrcScene *s; const MrtRay *rays; MrtHit *hits; const float *dist; uint8_t *occ; } TraceJob;
static void closest_body(long i, void *vctx, uint64_t *cnt) {
    TraceJob *j = (TraceJob *)vctx;
    const Ray r = ray_from(&j->rays[i]);
    Isect it;
    if (scene_closest(j->s, &r, &it)) { j->hits[i].t = it.length; j->hits[i].id = it.id; }
    else { j->hits[i].t = RAY_LENGTH_MAX; j->hits[i].id = MRT_HIT_NONE; }
}
static void any_body(long i, void *vctx, uint64_t *cnt) {
    TraceJob *j = (TraceJob *)vctx;
    const Ray r = ray_from(&j->rays[i]);
    j->occ[i] = (uint8_t)scene_occ(j->s, &r, j->dist[i]);
}
void orc_trace_closest(OrcScene *s, const MrtRay *rays, uint32_t n, MrtHit *hits, int threads) {
    TraceJob j; j.s = s; j.rays = rays; j.hits = hits; j.dist = NULL; j.occ = NULL;
    par_for((long)n, threads, 16, closest_body, &j, NULL);
}
void orc_trace_any(OrcScene *s, const MrtRay *rays, const float *dist, uint32_t n, uint8_t *occ, int threads) {
    TraceJob j; j.s = s; j.rays = rays; j.hits = NULL; j.dist = dist; j.occ = occ;
    par_for((long)n, threads, 16, any_body, &j, NULL);
}

/* the grid walk's work per ray: cells visited and triangle references tested in the triangle grid,
 * after the plane and sphere grids (the counting replay of the device grid walk) */
typedef struct { OrcScene *s; const MrtRay *rays; uint32_t *cells, *refs; } CountJob;
static void count_body(long i, void *vctx, uint64_t *cnt) {
    CountJob *j = (CountJob *)vctx;
    const Ray r = ray_from(&j->rays[i]);
    Isect it;
    it.length = RAY_LENGTH_MAX; it.id = MRT_HIT_NONE; it.light = -1; it.mat = 0;
    grid_trace(&j->s->grid[T_PLANE], &j->s->sets[T_PLANE], &r, &it);
    grid_trace(&j->s->grid[T_SPHERE], &j->s->sets[T_SPHERE], &r, &it);
    j->cells[i] = 0;
    j->refs[i] = 0;
    grid_trace_n(&j->s->grid[T_TRI], &j->s->sets[T_TRI], &r, &it, &j->cells[i], &j->refs[i]);
}
int orc_grid_counts(OrcScene *s, const MrtRay *rays, uint32_t n, uint32_t *cells, uint32_t *refs, int threads) {
    if (s->accel != ORC_ACCEL_GRID) return 1;
    CountJob j; j.s = s; j.rays = rays; j.cells = cells; j.refs = refs;
    par_for((long)n, threads, 16, count_body, &j, NULL);
    return 0;
}

/* ============================== keyed stream and samplers ===================================== */
/* 32-bit avalanche mixer (Wellons' "lowbias32", hash-prospector, published constants) */
static inline uint32_t mix32(uint32_t x) {
    x ^= x >> 16; x *= 0x21f0aaadu; x ^= x >> 15; x *= 0x735a2d97u; x ^= x >> 15; return x;
}
static inline uint32_t key_base(uint64_t seed, uint32_t pixel, uint32_t sample) {
    uint32_t h = mix32((uint32_t)seed ^ 0x9e3779b9u);
    h = mix32(h ^ (uint32_t)(seed >> 32));
    h = mix32(h ^ pixel);
    return mix32(h ^ sample);
}
static inline float key_float(uint32_t base, uint32_t node, uint32_t dim) {
    const uint32_t h = mix32(mix32(base ^ node) ^ dim);
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}
/* Halton base of dimension dim: the dim-th prime (dims 0-1 camera, 2 roulette, 8 + 3j + 1..2 light
 * sample j < 32 all lie below 128, so no two dimensions share a base) */
#define HALTON_DIMS 128u
static const uint32_t PRIMES[HALTON_DIMS] = {
    2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
    59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127, 131,
    137, 139, 149, 151, 157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223,
    227, 229, 233, 239, 241, 251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311,
    313, 317, 331, 337, 347, 349, 353, 359, 367, 373, 379, 383, 389, 397, 401, 409,
    419, 421, 431, 433, 439, 443, 449, 457, 461, 463, 467, 479, 487, 491, 499, 503,
    509, 521, 523, 541, 547, 557, 563, 569, 571, 577, 587, 593, 599, 601, 607, 613,
    617, 619, 631, 641, 643, 647, 653, 659, 661, 673, 677, 683, 691, 701, 709, 719,
};

/* haltonSequence  Utils.cpp:36-45 */
float orc_halton(uint32_t index, uint32_t base) {
    float f = 1.0f, result = 0.0f;
    while (index > 0) {
        f /= (float)base;
        result += f * (float)(index % base);
        index = index / base;
    }
    return result;
}

typedef struct {
    const MrtRenderOpts *o;
    uint32_t pixel, sample;
    uint32_t base;       /* key_base(seed, pixel, sample) */
    uint32_t rot_base;   /* key_base(seed, pixel, 0xFFFFFFFF): sample-independent rotations */
    uint64_t n_closest, n_shadow;
} Stream;

static float stream_draw(const Stream *st, int kind, uint32_t node, uint32_t dim) {
    switch (kind) {
        case MRT_SAMPLER_CONSTANT: return st->o->constant_value;
        case MRT_SAMPLER_STRATIFIED: {
            float v = (float)st->sample / (float)(st->o->spp > 0 ? st->o->spp : 1) + key_float(st->rot_base, node, dim);
            if (v >= 1.0f) v -= 1.0f;
            return v;
        }
        case MRT_SAMPLER_HALTON: {
            float v = orc_halton(st->sample, PRIMES[dim % HALTON_DIMS]) + key_float(st->rot_base, node, dim);
            if (v >= 1.0f) v -= 1.0f;
            return v;
        }
        default: return key_float(st->base, node, dim);
    }
}

float orc_sample(const MrtRenderOpts *o, int kind, uint32_t pixel, uint32_t sample, uint32_t node, uint32_t dim) {
    Stream st; memset(&st, 0, sizeof(st));
    st.o = o; st.pixel = pixel; st.sample = sample;
    st.base = key_base(o->seed, pixel, sample);
    st.rot_base = key_base(o->seed, pixel, 0xFFFFFFFFu);
    return stream_draw(&st, kind, node, dim);
}

/* Stream dimensions: 0,1 camera jitter (node 0); per shaded node: 2 Russian roulette,
 * 3,4 hemisphere, 8+3j light choice, 9+3j / 10+3j area-light R / S of light sample j. */
#define DIM_RR 2u
#define DIM_HEMI 3u
#define DIM_LIGHT 8u

/* sin and cos of x in [0, 2*pi): quadrant reduction by a two-part pi/2 (Cody-Waite) and Taylor
 * polynomials to degree 9 / 10 on [-pi/4, pi/4], plain float multiplies and adds only, so the CPU
 * and the GPU produce the same bits.  (The reference calls std::sin / std::cos, Shader.cpp:217-219.) */
void orc_sincos(float x, float *s_out, float *c_out) {
    const float two_over_pi = 0.636619772367581343f;
    const float pio2_hi = 1.5703125f;                 /* 201/128, exact in float */
    const float pio2_lo = 4.83826794897e-4f;          /* pi/2 - pio2_hi */
    float kf = x * two_over_pi + 0.5f;
    const int32_t k = (int32_t)kf;
    kf = (float)k;
    const float r = (x - kf * pio2_hi) - kf * pio2_lo;
    const float r2 = r * r;
    const float sp = r + r * r2 * (-1.0f / 6.0f + r2 * (1.0f / 120.0f + r2 * (-1.0f / 5040.0f + r2 * (1.0f / 362880.0f))));
    const float cp = 1.0f + r2 * (-0.5f + r2 * (1.0f / 24.0f + r2 * (-1.0f / 720.0f + r2 * (1.0f / 40320.0f + r2 * (-1.0f / 3628800.0f)))));
    switch (k & 3) {
        case 0: *s_out = sp; *c_out = cp; break;
        case 1: *s_out = cp; *c_out = -sp; break;
        case 2: *s_out = -sp; *c_out = -cp; break;
        default: *s_out = -cp; *c_out = sp; break;
    }
}

/* Shader::getCosineSampleHemisphere  Shader.cpp:193-223 with stream draws */
static V3 hemisphere(V3 n, float u1, float u2) {
    const float phi = 6.28318530717958647692f * u1;
    const float r2 = u2;
    const float cos_theta = sqrtf(r2);
    V3 u = fabsf(n.x) > 0.1f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    u = vnormalize(vcross(u, n));
    const V3 v = vcross(n, u);
    float sp, cp;
    orc_sincos(phi, &sp, &cp);
    V3 dir = vadd(vadd(vscale(u, cp * cos_theta), vscale(v, sp * cos_theta)), vscale(n, sqrtf(1.0f - r2)));
    return vnormalize(dir);
}

/* ============================== camera  Camera.cpp:52-57, Perspective.cpp:10-44 =============== */
typedef struct { V3 position, direction, right, up; float hfov, vfov; int kind; } Cam;
static Cam cam_make(const MrtCamera *c) {
    Cam k;
    k.position = vld(c->position);
    k.direction = vnormalize(vsub(vld(c->look_at), k.position));
    k.right = vcross(vld(c->up), k.direction);
    k.up = vcross(k.direction, k.right);
    k.kind = c->kind;
    if (c->kind == MRT_CAMERA_ORTHOGRAPHIC) {   /* Orthographic.cpp:12-17 */
        k.hfov = c->fov_h_deg / 2.0f;
        k.vfov = c->fov_v_deg / 2.0f;
        return k;
    }
    const float pi = 3.14159265358979323846f;
    k.hfov = (c->fov_h_deg * pi) / 180.0f;
    k.vfov = (c->fov_v_deg * pi) / 180.0f;
    return k;
}
static float fast_arctan(float x) {
    const float ax = fabsf(x);
    return 0.785398163397448309616f * x - (x * (ax - 1.0f)) * (0.2447f + (0.0663f * ax));
}
static Ray cam_ray(const Cam *k, float u, float v, float du, float dv) {
    if (k->kind == MRT_CAMERA_ORTHOGRAPHIC) {   /* Orthographic::generateRay  Orthographic.cpp:23-34 */
        const V3 right = vadd(vscale(k->right, (u - 0.5f) * k->hfov), vscale(k->right, du));
        const V3 up = vadd(vscale(k->up, (0.5f - v) * k->vfov), vscale(k->up, dv));
        Ray r; r.dir = k->direction; r.origin = vadd(vadd(k->position, right), up); r.depth = 1; r.exclude = MRT_HIT_NONE;
        return r;
    }
    const float rf = fast_arctan(k->hfov * (u - 0.5f)) + du;
    const V3 right = vscale(k->right, rf);
    const float uf = fast_arctan(k->vfov * (0.5f - v)) + dv;
    const V3 up = vscale(k->up, uf);
    const V3 dest = vadd(vadd(vadd(k->position, k->direction), right), up);
    Ray r; r.dir = vnormalize(vsub(dest, k->position)); r.origin = k->position; r.depth = 1; r.exclude = MRT_HIT_NONE;
    return r;
}
/* Camera::getAABB (Camera.cpp:39-44) / Orthographic::getAABB (Orthographic.cpp:36-46) */
void orc_camera_box(const MrtCamera *c, float *mn, float *mx) {
    const Cam k = cam_make(c);
    V3 a = k.position, b = k.position;
    if (c->kind == MRT_CAMERA_ORTHOGRAPHIC) {
        a = vadd(vadd(vadd(vadd(k.position, vscale(vscale(k.right, 0.0f - 0.5f), k.hfov)), vscale(k.right, -0.5f)),
                      vscale(vscale(k.up, 0.5f - 0.0f), k.vfov)), vscale(k.up, -0.5f));
        b = vadd(vadd(vadd(vadd(k.position, vscale(vscale(k.right, 1.0f - 0.5f), k.hfov)), vscale(k.right, 0.5f)),
                      vscale(vscale(k.up, 0.5f - 1.0f), k.vfov)), vscale(k.up, 0.5f));
    }
    mn[0] = a.x; mn[1] = a.y; mn[2] = a.z;
    mx[0] = b.x; mx[1] = b.y; mx[2] = b.z;
}

void orc_camera_ray(const MrtCamera *c, float u, float v, float du, float dv, float *o6) {
    const Cam k = cam_make(c);
    const Ray r = cam_ray(&k, u, v, du, dv);
    o6[0] = r.origin.x; o6[1] = r.origin.y; o6[2] = r.origin.z;
    o6[3] = r.dir.x; o6[4] = r.dir.y; o6[5] = r.dir.z;
}

/* ============================== shaders ======================================================= */
typedef struct { const OrcScene *s; Stream *st; } Ctx;

static int ray_trace(Ctx *c, V3 *rgb, const Ray *r, uint32_t node);

/* Shader::getLight  Shader.cpp:225-236 */
static const Lgt *pick_light(Ctx *c, uint32_t node, uint32_t j) {
    const float u = key_float(c->st->base, node, DIM_LIGHT + 3u * j);
    const uint32_t n = c->s->n_light;
    const uint32_t k = (uint32_t)floorf(u * (float)n * 0.99999f);
    return &c->s->light[k];
}
/* Light::getPosition: PointLight.cpp:17-19, AreaLight.cpp:22-31 */
static V3 light_position(Ctx *c, const Lgt *l, uint32_t node, uint32_t j) {
    if (l->kind != MRT_LIGHT_AREA) return l->pos;
    float R = stream_draw(c->st, c->st->o->light_sampler, node, DIM_LIGHT + 3u * j + 1u);
    float S = stream_draw(c->st, c->st->o->light_sampler, node, DIM_LIGHT + 3u * j + 2u);
    if (R + S >= 1.0f) { R = 1.0f - R; S = 1.0f - S; }
    return vadd(vadd(l->tri.a, vscale(l->tri.ab, R)), vscale(l->tri.ac, S));
}

static int material_of(const OrcScene *s, const Isect *it, Mat *m) {
    if (it->light >= 0) { *m = s->light[it->light].radiance; return 1; }
    if (it->mat >= 0) { *m = s->mat[it->mat]; return 1; }
    return 0;
}

/* direct light with shadow rays, shared by Whitted (Whitted.cpp:33-66) and PathTracer (:71-103) */
static V3 direct_shadowed(Ctx *c, const Isect *it, const Ray *r, V3 kd, uint32_t node) {
    V3 acc = v3(0, 0, 0);
    const uint32_t spl = c->st->o->spl;
    for (uint32_t j = 0; j < spl; ++j) {
        const Lgt *l = pick_light(c, node, j);
        const V3 lp = light_position(c, l, node, j);
        V3 vtl = vsub(lp, it->point);
        const float dist = vlength(vtl);
        vtl = vnormalize(vtl);
        const float cosnl = vdot(it->normal, vtl);
        if (cosnl > 0.0f) {
            Ray sr; sr.origin = it->point; sr.dir = vtl; sr.depth = r->depth + 1; sr.exclude = it->prim;
            c->st->n_shadow++;
            if (!scene_occ(c->s, &sr, dist)) acc = vadd(acc, vscale(l->radiance.le, cosnl));
        }
    }
    acc = vmul(acc, kd);
    return vdivs(acc, (float)spl);
}

/* NoShadows::shade  NoShadows.cpp:19-65 */
static int shade_noshadows(Ctx *c, V3 *rgb, const Isect *it, uint32_t node) {
    V3 kd;
    Mat m;
    if (material_of(c->s, it, &m)) {
        if (vany_pos(m.le)) { *rgb = m.le; return 1; }
        kd = m.kd;
    } else kd = it->color;
    if (vany_pos(kd) && c->s->n_light > 0) {
        const uint32_t spl = c->st->o->spl;
        for (uint32_t j = 0; j < spl; ++j) {
            const Lgt *l = pick_light(c, node, j);
            const V3 lp = light_position(c, l, node, j);
            const V3 vtl = vnormalize(vsub(lp, it->point));
            const float cosnl = vdot(it->normal, vtl);
            if (cosnl > 0.0f) *rgb = vadd(*rgb, vscale(l->radiance.le, cosnl));
        }
        *rgb = vmul(*rgb, kd);
        *rgb = vdivs(*rgb, (float)spl);
    }
    *rgb = vadd(*rgb, vscale(kd, 0.1f));
    return 0;
}

/* Whitted::shade  Whitted.cpp:17-107 */
static int shade_whitted(Ctx *c, V3 *rgb, const Isect *it, const Ray *r, uint32_t node) {
    if (r->depth > c->st->o->depth_max) return 0;
    V3 kd, ks = v3(0, 0, 0), kt = v3(0, 0, 0);
    float ior = 1.0f;
    Mat m;
    if (material_of(c->s, it, &m)) {
        if (vany_pos(m.le)) { *rgb = m.le; return 1; }
        kd = m.kd; ks = m.ks; kt = m.kt; ior = m.ior;
    } else kd = it->color;
    if (vany_pos(kd) && c->s->n_light > 0) {
        const uint32_t spl = c->st->o->spl;
        for (uint32_t j = 0; j < spl; ++j) {
            const Lgt *l = pick_light(c, node, j);
            const V3 lp = light_position(c, l, node, j);
            V3 vtl = vsub(lp, it->point);
            const float dist = vlength(vtl);
            vtl = vnormalize(vtl);
            const float cosnl = vdot(it->normal, vtl);
            if (cosnl > 0.0f) {
                Ray sr; sr.origin = it->point; sr.dir = vtl; sr.depth = r->depth + 1; sr.exclude = it->prim;
                c->st->n_shadow++;
                if (!scene_occ(c->s, &sr, dist)) *rgb = vadd(*rgb, vscale(l->radiance.le, cosnl));
            }
        }
        *rgb = vmul(*rgb, kd);
        *rgb = vdivs(*rgb, (float)spl);
    }
    if (vany_pos(ks)) {
        Ray sr; sr.origin = it->point; sr.dir = vreflect(r->dir, it->normal); sr.depth = r->depth + 1; sr.exclude = it->prim;
        V3 lis = v3(0, 0, 0);
        ray_trace(c, &lis, &sr, node * 4u + 2u);
        *rgb = vadd(*rgb, vmul(ks, lis));
    }
    if (vany_pos(kt)) {
        Ray tr; tr.origin = it->point; tr.dir = vrefract(r->dir, it->normal, 1.0f / ior); tr.depth = r->depth + 1; tr.exclude = it->prim;
        V3 lit = v3(0, 0, 0);
        ray_trace(c, &lit, &tr, node * 4u + 3u);
        *rgb = vadd(*rgb, vmul(kt, lit));
    }
    *rgb = vadd(*rgb, vscale(kd, 0.1f));
    return 0;
}

/* PathTracer::shade  PathTracer.cpp:25-164 */
static int shade_pathtracer(Ctx *c, V3 *rgb, const Isect *it, const Ray *r, uint32_t node) {
    const int32_t depth = r->depth;
    if (depth > c->st->o->depth_max) return 0;
    V3 kd, ks = v3(0, 0, 0), kt = v3(0, 0, 0);
    float ior = 1.0f;
    Mat m;
    if (material_of(c->s, it, &m)) {
        if (vany_pos(m.le)) { *rgb = m.le; return 1; }
        kd = m.kd; ks = m.ks; kt = m.kt; ior = m.ior;
    } else kd = it->color;
    V3 ld = v3(0, 0, 0), lid = v3(0, 0, 0), lis = v3(0, 0, 0), lit = v3(0, 0, 0);
    int hit_light = 0;
    if (vany_pos(kd)) {
        if (c->s->n_light > 0) ld = direct_shadowed(c, it, r, kd, node);
        int go = depth <= c->st->o->depth_min;
        if (!go) go = stream_draw(c->st, c->st->o->rr_sampler, node, DIM_RR) > 0.5f;
        if (go) {
            const float u1 = key_float(c->st->base, node, DIM_HEMI), u2 = key_float(c->st->base, node, DIM_HEMI + 1u);
            Ray nr; nr.origin = it->point; nr.dir = hemisphere(it->normal, u1, u2); nr.depth = depth + 1; nr.exclude = it->prim;
            V3 child = v3(0, 0, 0);
            hit_light = ray_trace(c, &child, &nr, node * 4u + 1u);
            lid = vadd(lid, vmul(kd, child));
            if (depth > c->st->o->depth_min) lid = vdivs(lid, 0.5f * 0.5f);
            if (vany_pos(ld) && hit_light) lid = v3(0, 0, 0);
        }
    }
    if (vany_pos(ks)) {
        Ray sr; sr.origin = it->point; sr.dir = vreflect(r->dir, it->normal); sr.depth = depth + 1; sr.exclude = it->prim;
        V3 child = v3(0, 0, 0);
        ray_trace(c, &child, &sr, node * 4u + 2u);
        lis = vadd(lis, vmul(ks, child));
    }
    if (vany_pos(kt)) {
        Ray tr; tr.origin = it->point; tr.dir = vrefract(r->dir, it->normal, 1.0f / ior); tr.depth = depth + 1; tr.exclude = it->prim;
        V3 child = v3(0, 0, 0);
        ray_trace(c, &child, &tr, node * 4u + 3u);
        lit = vadd(lit, vmul(kt, child));
    }
    *rgb = vadd(*rgb, ld);
    *rgb = vadd(*rgb, lid);
    *rgb = vadd(*rgb, lis);
    *rgb = vadd(*rgb, lit);
    return hit_light;
}

/* Shader::rayTrace  Shader.cpp:124-160 */
/* DepthMap::shade  DepthMap.cpp:19-26 */
static int shade_depthmap(Ctx *c, V3 *rgb, const Isect *it, const Ray *r) {
    const float max_dist = vlength(vsub(vld(c->st->o->depth_point), r->origin)) * 2.0f;
    const float x = (max_dist - it->length) / max_dist;
    const float depth = x < 0.0f ? 0.0f : x;   /* std::max(x, 0.0f) */
    *rgb = v3(depth, depth, depth);
    return 0;
}

/* DiffuseMaterial::shade  DiffuseMaterial.cpp:16-38 */
static int shade_diffuse(Ctx *c, V3 *rgb, const Isect *it) {
    Mat m;
    if (material_of(c->s, it, &m)) {
        if (vany_pos(m.kd)) *rgb = m.kd;
        else if (vany_pos(m.ks)) *rgb = m.ks;
        else if (vany_pos(m.kt)) *rgb = m.kt;
        else if (vany_pos(m.le)) *rgb = m.le;
    } else {
        *rgb = it->color;
    }
    return 0;
}

static int ray_trace(Ctx *c, V3 *rgb, const Ray *r, uint32_t node) {
    Isect it;
    c->st->n_closest++;
    if (!scene_closest(c->s, r, &it)) return 0;
    switch (c->st->o->shader) {
        case MRT_SHADER_DEPTHMAP: return shade_depthmap(c, rgb, &it, r);
        case MRT_SHADER_DIFFUSE: return shade_diffuse(c, rgb, &it);
        case MRT_SHADER_WHITTED: return shade_whitted(c, rgb, &it, r, node);
        case MRT_SHADER_PATHTRACER: return shade_pathtracer(c, rgb, &it, r, node);
        default: return shade_noshadows(c, rgb, &it, node);
    }
}

/* ============================== renderer  Renderer.cpp ======================================== */
/* float -> uint32 as the reference build does it on x86-64 (truncate through a 64-bit signed
 * register, keep the low 32 bits; NaN and out-of-range give 0), Utils.cpp:56-58 */
static uint32_t f2u_x86(float f) {
    if (!(f > -9.2233720368547758e18f && f < 9.2233720368547758e18f)) return 0u;
    return (uint32_t)(int64_t)f;
}

/* incrementalAvg  Utils.cpp:48-70 */
uint32_t orc_incremental_avg(const float *rgb, uint32_t avg, uint32_t n) {
    const uint32_t lr = avg & 0xFFu, lg = (avg >> 8u) & 0xFFu, lb = (avg >> 16u) & 0xFFu;
    const uint32_t sr = f2u_x86(rgb[0] * 255.0f), sg = f2u_x86(rgb[1] * 255.0f), sb = f2u_x86(rgb[2] * 255.0f);
    const uint32_t cr = ((n - 1u) * lr + sr) / n, cg = ((n - 1u) * lg + sg) / n, cb = ((n - 1u) * lb + sb) / n;
    const uint32_t rr = cr < 255u ? cr : 255u, rg = cg < 255u ? cg : 255u, rb = cb < 255u ? cb : 255u;
    return 0xFF000000u | (rb << 16u) | (rg << 8u) | rr;
}

float orc_aabb_area(const float *bmin, const float *bmax) { Box b; b.mn = vld(bmin); b.mx = vld(bmax); return box_area(&b); }

/* one camera sample of one pixel: Renderer.cpp:94-104 */
static V3 pixel_sample(const OrcScene *s, const Cam *cam, const MrtRenderOpts *o, uint32_t x, uint32_t y,
                       uint32_t sample, uint64_t *nc, uint64_t *ns) {
    Stream st; memset(&st, 0, sizeof(st));
    st.o = o;
    st.pixel = y * o->width + x;
    st.sample = sample;
    st.base = key_base(o->seed, st.pixel, sample);
    st.rot_base = key_base(o->seed, st.pixel, 0xFFFFFFFFu);
    const float inv_w = 1.0f / (float)o->width, inv_h = 1.0f / (float)o->height;
    const float pw = 0.5f / (float)o->width, ph = 0.5f / (float)o->height;
    const float u = (float)x * inv_w, v = (float)y * inv_h;
    const float r1 = stream_draw(&st, o->pixel_sampler, 0u, 0u);
    const float r2 = stream_draw(&st, o->pixel_sampler, 0u, 1u);
    const Ray r = cam_ray(cam, u, v, (r1 - 0.5f) * 2.0f * pw, (r2 - 0.5f) * 2.0f * ph);
    V3 rgb = v3(0, 0, 0);
    Ctx c; c.s = s; c.st = &st;
    ray_trace(&c, &rgb, &r, 1u);
    if (nc) *nc += st.n_closest;
    if (ns) *ns += st.n_shadow;
    return rgb;
}

typedef struct { uint32_t x, y, index; } Task;

/* the pixels one sample pass visits, in block order i = 0..255 (the reference visits the same
 * blocks in a shuffled order, Camera.cpp:13-37, Renderer.cpp:79-93) */
static Task *block_tasks(uint32_t w, uint32_t h, uint32_t real_w, uint32_t *count) {
    const uint32_t bsx = w / 16u, bsy = h / 16u;   /* Renderer.cpp:20-21 */
    const uint32_t domain = (w / bsx) * (h / bsy);
    const uint32_t res = w * h;
    size_t cap = (size_t)NUMBER_OF_BLOCKS * bsx * bsy, n = 0;
    Task *t = malloc(sizeof(Task) * (cap ? cap : 1));
    for (uint32_t i = 0; i < NUMBER_OF_BLOCKS; ++i) {
        const float block = orc_halton(i, 2);
        const uint32_t rb = (uint32_t)roundf(block * (float)domain);
        const uint32_t pixel = rb * bsx % res;
        const uint32_t sy = ((pixel / w) * bsy) % h;
        for (uint32_t y = sy; y < sy + bsy; ++y) {
            const uint32_t yw = y * real_w;
            const uint32_t sx = (pixel + yw) % w;
            for (uint32_t x = sx; x < sx + bsx; ++x) { t[n].x = x; t[n].y = y; t[n].index = yw + x; ++n; }
        }
    }
    *count = (uint32_t)n;
    return t;
}

typedef struct { const OrcScene *s; const Cam *cam; const MrtRenderOpts *o; const Task *tasks; uint32_t *bitmap; float *accum; uint32_t sample; uint32_t real_w; } RenderJob;
static void render_body(long k, void *vctx, uint64_t *cnt) {
    RenderJob *j = (RenderJob *)vctx;
    const Task *t = &j->tasks[k];
    const V3 rgb = pixel_sample(j->s, j->cam, j->o, t->x, t->y, j->sample, &cnt[0], &cnt[1]);
    const float c3[3] = {rgb.x, rgb.y, rgb.z};
    j->bitmap[t->index] = orc_incremental_avg(c3, j->bitmap[t->index], j->sample + 1u);
    const uint32_t row = t->index / j->real_w, col = t->index % j->real_w;
    if (j->accum && col < j->o->width) {
        float *a = j->accum + 4 * ((size_t)row * j->o->width + col);
        a[0] += rgb.x; a[1] += rgb.y; a[2] += rgb.z; a[3] += 1.0f;
    }
}

int orc_render(OrcScene *s, const MrtCamera *camera, const MrtRenderOpts *o, uint32_t *bitmap,
               uint32_t stride_bytes, float *accum, uint64_t *ray_counts, int threads) {
    if (o->width < 16 || o->height < 16) return MRT_ERR_ARG;
    const uint32_t real_w = stride_bytes / 4u;
    const Cam cam = cam_make(camera);
    uint32_t nt = 0;
    Task *tasks = block_tasks(o->width, o->height, real_w, &nt);
    /* pixels visited more than once per pass are processed in block order, one task at a time */
    uint8_t *seen = calloc((size_t)real_w * o->height + 1, 1);
    int dup = 0;
    for (uint32_t k = 0; k < nt; ++k) {
        if (tasks[k].index >= real_w * o->height) { dup = 1; continue; }
        if (seen[tasks[k].index]++) dup = 1;
    }
    free(seen);
    uint64_t nc = 0, ns = 0;
    if (threads < 1) threads = 1;
    for (uint32_t si = 0; si < o->spp; ++si) {
        const uint32_t sample = o->spp_offset + si;
        if (dup) {
            for (uint32_t k = 0; k < nt; ++k) {
                if (tasks[k].index >= real_w * o->height) continue;
                const V3 rgb = pixel_sample(s, &cam, o, tasks[k].x, tasks[k].y, sample, &nc, &ns);
                const float c3[3] = {rgb.x, rgb.y, rgb.z};
                bitmap[tasks[k].index] = orc_incremental_avg(c3, bitmap[tasks[k].index], sample + 1u);
                const uint32_t row = tasks[k].index / real_w, col = tasks[k].index % real_w;
                if (accum && col < o->width) {   /* the fp32 sum of the bitmap pixel written */
                    float *a = accum + 4 * ((size_t)row * o->width + col);
                    a[0] += rgb.x; a[1] += rgb.y; a[2] += rgb.z; a[3] += 1.0f;
                }
            }
        } else {
            RenderJob j; j.s = s; j.cam = &cam; j.o = o; j.tasks = tasks; j.bitmap = bitmap; j.accum = accum; j.sample = sample; j.real_w = real_w;
            uint64_t cnt[2];
            par_for((long)nt, threads, 64, render_body, &j, cnt);
            nc += cnt[0]; ns += cnt[1];
        }
    }
    free(tasks);
    if (ray_counts) { ray_counts[0] = nc; ray_counts[1] = ns; }
    return MRT_OK;
}

typedef struct { const OrcScene *s; const Cam *cam; const MrtRenderOpts *o; const uint32_t *xy; float *out; } PixJob;
static void pixels_body(long k, void *vctx, uint64_t *cnt) {
    PixJob *j = (PixJob *)vctx;
    for (uint32_t si = 0; si < j->o->spp; ++si) {
        const V3 rgb = pixel_sample(j->s, j->cam, j->o, j->xy[2 * k], j->xy[2 * k + 1], j->o->spp_offset + si, &cnt[0], &cnt[1]);
        float *p = j->out + ((size_t)k * j->o->spp + si) * 3;
        p[0] = rgb.x; p[1] = rgb.y; p[2] = rgb.z;
    }
}
int orc_render_pixels(OrcScene *s, const MrtCamera *camera, const MrtRenderOpts *o, const uint32_t *xy,
                      uint32_t n, float *out, int threads) {
    const Cam cam = cam_make(camera);
    PixJob j; j.s = s; j.cam = &cam; j.o = o; j.xy = xy; j.out = out;
    par_for((long)n, threads, 4, pixels_body, &j, NULL);
    return MRT_OK;
}

/* ============================== single-function entry points (KATs) =========================== */
int orc_triangle_intersect(const float *abc, const float *normals, const float *colors, const float *o,
                           const float *d, float length, float *out_t, float *out_normal, float *out_color) {
    const Tri t = tri_make(abc, normals, colors, -1);
    Ray r; r.origin = vld(o); r.dir = vld(d); r.depth = 1; r.exclude = MRT_HIT_NONE;
    Isect it; memset(&it, 0, sizeof(it)); it.length = length;
    const int hit = tri_hit(&t, 0u, &r, &it);
    if (out_t) *out_t = it.length;
    if (out_normal) { out_normal[0] = it.normal.x; out_normal[1] = it.normal.y; out_normal[2] = it.normal.z; }
    if (out_color) { out_color[0] = it.color.x; out_color[1] = it.color.y; out_color[2] = it.color.z; }
    return hit;
}
int orc_triangle_occludes(const float *abc, const float *o, const float *d, float dist) {
    const Tri t = tri_make(abc, NULL, NULL, -1);
    Ray r; r.origin = vld(o); r.dir = vld(d); r.depth = 1; r.exclude = MRT_HIT_NONE;
    return tri_occ(&t, 0u, &r, dist);
}
int orc_triangle_intersect_box(const float *abc, const float *bmin, const float *bmax) {
    const Tri t = tri_make(abc, NULL, NULL, -1);
    Box b; b.mn = vld(bmin); b.mx = vld(bmax);
    return tri_in_box(&t, &b);
}
int orc_plane_intersect_box(const float *pn, const float *bmin, const float *bmax) {
    const Pln p = pln_make(pn, -1);
    Box b; b.mn = vld(bmin); b.mx = vld(bmax);
    return pln_in_box(&p, &b);
}
float orc_plane_distance(const float *pn, const float *q) { const Pln p = pln_make(pn, -1); return pln_distance(&p, vld(q)); }
int orc_plane_intersect(const float *pn, const float *o, const float *d, float length, float *out_t) {
    const Pln p = pln_make(pn, -1);
    Ray r; r.origin = vld(o); r.dir = vld(d); r.depth = 1; r.exclude = MRT_HIT_NONE;
    Isect it; memset(&it, 0, sizeof(it)); it.length = length;
    const int hit = pln_hit(&p, 0u, &r, &it);
    *out_t = it.length;
    return hit;
}
int orc_sphere_intersect(const float *cr, const float *o, const float *d, float length, float *out_t, float *out_n) {
    const Sph s = sph_make(cr, -1);
    Ray r; r.origin = vld(o); r.dir = vld(d); r.depth = 1; r.exclude = MRT_HIT_NONE;
    Isect it; memset(&it, 0, sizeof(it)); it.length = length;
    const int hit = sph_hit(&s, 0u, &r, &it);
    *out_t = it.length;
    if (out_n) { out_n[0] = it.normal.x; out_n[1] = it.normal.y; out_n[2] = it.normal.z; }
    return hit;
}
int orc_sphere_intersect_box(const float *cr, const float *bmin, const float *bmax) {
    const Sph s = sph_make(cr, -1);
    Box b; b.mn = vld(bmin); b.mx = vld(bmax);
    return sph_in_box(&s, &b);
}
int orc_aabb_intersect(const float *bmin, const float *bmax, const float *o, const float *d) {
    Box b; b.mn = vld(bmin); b.mx = vld(bmax);
    Ray r; r.origin = vld(o); r.dir = vld(d); r.depth = 1; r.exclude = MRT_HIT_NONE;
    return box_hit(&b, &r);
}

/* ================================ raster preview ==================================================
 * The Android front end's first image (MainRenderer.copyFrame, MainRenderer.java:338-546, over
 * DrawView.cpp:47-210 and VertexShaderRaster.glsl / FragmentShaderRaster.glsl): the scene triangles
 * (A, A + AB, A + AC with z negated, DrawView.cpp:131-154), one colour each (DrawView.cpp:178-196),
 * projection x view from android.opengl.Matrix (perspectiveM with fovY = 0.918 x the vertical field
 * of view, near 0.1, far 1e38, or orthoM with the film half sizes; setLookAtM on the z-negated
 * camera), back faces culled (CCW front), depth test LEQUAL against 1, colour cleared to 0, rows
 * flipped on read-back (copyFrameBuffer, MainRenderer.java:111-139).  The steps OpenGL leaves to the
 * implementation are the library's (clip near/far and a guard band of 16 w in x and y, snap to 1/256
 * pixel, pixel centres with the top-left rule, linear window-space depth clamped to [0, 1]); this is
 * an independent serial restatement with a literal LEQUAL depth buffer in draw order. */
typedef struct { float m[16]; } M4;   /* column-major: (row r, column c) at m[4 c + r] */
/* clipped polygon: at most 9 vertices in exact arithmetic; rounding can make it slightly non-convex
 * and let a later plane add more, so there is room for 16 and vertices beyond that are dropped */
#define RAS_MAX_POLY 16
typedef struct { float x, y, z, w; } C4;

static M4 m4_perspective(float fovy, float aspect, float zn, float zf) {
    M4 r; memset(&r, 0, sizeof(r));
    const float f = 1.0f / (float)tan((double)fovy * (3.14159265358979323846 / 360.0));
    const float rr = 1.0f / (zn - zf);
    r.m[0] = f / aspect; r.m[5] = f; r.m[10] = (zf + zn) * rr; r.m[11] = -1.0f; r.m[14] = 2.0f * zf * zn * rr;
    return r;
}
static M4 m4_ortho(float l, float rt, float b, float t, float zn, float zf) {
    M4 r; memset(&r, 0, sizeof(r));
    const float rw = 1.0f / (rt - l), rh = 1.0f / (t - b), rd = 1.0f / (zf - zn);
    r.m[0] = 2.0f * rw; r.m[5] = 2.0f * rh; r.m[10] = -2.0f * rd;
    r.m[12] = -(rt + l) * rw; r.m[13] = -(t + b) * rh; r.m[14] = -(zf + zn) * rd; r.m[15] = 1.0f;
    return r;
}
static float m4_len(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }
static M4 m4_look_at(V3 e, V3 c, V3 u) {
    V3 f = vsub(c, e);
    const float rlf = 1.0f / m4_len(f.x, f.y, f.z);
    f = v3(f.x * rlf, f.y * rlf, f.z * rlf);
    V3 s = v3(f.y * u.z - f.z * u.y, f.z * u.x - f.x * u.z, f.x * u.y - f.y * u.x);
    const float rls = 1.0f / m4_len(s.x, s.y, s.z);
    s = v3(s.x * rls, s.y * rls, s.z * rls);
    const V3 v = v3(s.y * f.z - s.z * f.y, s.z * f.x - s.x * f.z, s.x * f.y - s.y * f.x);
    M4 r; memset(&r, 0, sizeof(r));
    r.m[0] = s.x; r.m[1] = v.x; r.m[2] = -f.x;
    r.m[4] = s.y; r.m[5] = v.y; r.m[6] = -f.y;
    r.m[8] = s.z; r.m[9] = v.z; r.m[10] = -f.z;
    r.m[15] = 1.0f;
    for (int i = 0; i < 4; ++i) r.m[12 + i] += r.m[i] * -e.x + r.m[4 + i] * -e.y + r.m[8 + i] * -e.z;   /* translateM */
    return r;
}
static M4 m4_mul(const M4 *a, const M4 *b) {
    M4 r;
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            r.m[4 * c + row] = ((a->m[row] * b->m[4 * c] + a->m[4 + row] * b->m[4 * c + 1]) + a->m[8 + row] * b->m[4 * c + 2]) +
                               a->m[12 + row] * b->m[4 * c + 3];
    return r;
}
static C4 ras_clip(const M4 *m, V3 p) {
    C4 c;
    c.x = ((m->m[0] * p.x + m->m[4] * p.y) + m->m[8] * p.z) + m->m[12];
    c.y = ((m->m[1] * p.x + m->m[5] * p.y) + m->m[9] * p.z) + m->m[13];
    c.z = ((m->m[2] * p.x + m->m[6] * p.y) + m->m[10] * p.z) + m->m[14];
    c.w = ((m->m[3] * p.x + m->m[7] * p.y) + m->m[11] * p.z) + m->m[15];
    return c;
}
static float ras_plane(C4 v, int p) {
    switch (p) {
        case 0: return v.z + v.w;
        case 1: return v.w - v.z;
        case 2: return 16.0f * v.w - v.x;
        case 3: return 16.0f * v.w + v.x;
        case 4: return 16.0f * v.w - v.y;
        default: return 16.0f * v.w + v.y;
    }
}
static int64_t ras_edge(int64_t xa, int64_t ya, int64_t xb, int64_t yb, int64_t px, int64_t py) {
    return (xb - xa) * (py - ya) - (yb - ya) * (px - xa);
}
static int ras_owns(int64_t xa, int64_t ya, int64_t xb, int64_t yb) { return yb < ya || (yb == ya && xb < xa); }
static int64_t ras_floor256(int64_t a) { return a >= 0 ? a / 256 : -((-a + 255) / 256); }
static uint32_t ras_unorm8(float c) {
    const float k = c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
    return (uint32_t)(k * 255.0f + 0.5f);
}

int orc_raster_preview(const MrtSceneDesc *d, const MrtCamera *cam, uint32_t width, uint32_t height, uint32_t *bitmap,
                       uint32_t stride_bytes, uint64_t *counts) {
    if (!d || !cam || !bitmap || width == 0 || height == 0 || stride_bytes < 4u * width) return 1;
    const Cam k = cam_make(cam);
    const V3 eye = v3(k.position.x, k.position.y, -k.position.z);
    const V3 dir = v3(k.direction.x, k.direction.y, -k.direction.z);
    const V3 up = v3(k.up.x, k.up.y, -k.up.z);
    M4 proj;
    if (cam->kind == MRT_CAMERA_ORTHOGRAPHIC) {
        proj = m4_ortho(-k.hfov / 2, k.hfov / 2, -k.vfov / 2, k.vfov / 2, 0.1f, 1.0e38f);
    } else {
        const float pi = 3.14159265358979323846f;
        const float w = (float)width, h = (float)height;
        const float ratio = (w / h) < (h / w) ? (h / w) : (w / h);
        const float hf = width > height ? ratio : 1.0f, vf = width < height ? ratio : 1.0f;
        float fovy = (k.vfov / pi) * 180.0f;
        fovy *= 0.918f;
        proj = m4_perspective(fovy, hf > vf ? hf : 1.0f / vf, 0.1f, 1.0e38f);
    }
    const M4 view = m4_look_at(eye, vadd(eye, dir), up);
    const M4 m = m4_mul(&proj, &view);
    const size_t npx = (size_t)width * height;
    float *depth = (float *)malloc(sizeof(float) * npx);
    int64_t *win = (int64_t *)malloc(sizeof(int64_t) * npx);
    if (!depth || !win) { free(depth); free(win); return 2; }
    for (size_t i = 0; i < npx; ++i) { depth[i] = 1.0f; win[i] = -1; }
    const float hw = 0.5f * (float)width, hh = 0.5f * (float)height;
    uint64_t drawn = 0, frags = 0;
    for (uint32_t i = 0; i < d->n_triangles; ++i) {
        const float *t = d->tri_abc + 9 * (size_t)i;
        const V3 A = vld(t), AB = vsub(vld(t + 3), A), AC = vsub(vld(t + 6), A);   /* Triangle.cpp: AB, AC */
        C4 poly[RAS_MAX_POLY], tmp[RAS_MAX_POLY];
        poly[0] = ras_clip(&m, v3(A.x, A.y, -A.z));
        poly[1] = ras_clip(&m, v3(A.x + AB.x, A.y + AB.y, -(A.z + AB.z)));
        poly[2] = ras_clip(&m, v3(A.x + AC.x, A.y + AC.y, -(A.z + AC.z)));
        int n = 3;
        for (int p = 0; p < 6 && n >= 3; ++p) {
            int out = 0;
            for (int q = 0; q < n; ++q) {
                const C4 S = poly[q], E = poly[(q + 1) % n];
                const float ds = ras_plane(S, p), de = ras_plane(E, p);
                if (ds >= 0.0f && out < RAS_MAX_POLY) tmp[out++] = S;
                if ((ds >= 0.0f) != (de >= 0.0f) && out < RAS_MAX_POLY) {
                    const float u = ds / (ds - de);
                    C4 c; c.x = S.x + u * (E.x - S.x); c.y = S.y + u * (E.y - S.y); c.z = S.z + u * (E.z - S.z);
                    c.w = S.w + u * (E.w - S.w);
                    tmp[out++] = c;
                }
            }
            n = out;
            memcpy(poly, tmp, sizeof(C4) * (size_t)n);
        }
        if (n < 3) continue;
        int64_t X[RAS_MAX_POLY], Y[RAS_MAX_POLY];
        float Z[RAS_MAX_POLY];
        for (int q = 0; q < n; ++q) {
            const float xn = poly[q].x / poly[q].w, yn = poly[q].y / poly[q].w, zn = poly[q].z / poly[q].w;
            X[q] = (int64_t)lrintf((hw * xn + hw) * 256.0f);
            Y[q] = (int64_t)lrintf((hh * yn + hh) * 256.0f);
            Z[q] = 0.5f * zn + 0.5f;
        }
        for (int f = 1; f + 1 < n; ++f) {
            const int v[3] = {0, f, f + 1};
            const int64_t x0 = X[v[0]], y0 = Y[v[0]], x1 = X[v[1]], y1 = Y[v[1]], x2 = X[v[2]], y2 = Y[v[2]];
            const float z0 = Z[v[0]], z1 = Z[v[1]], z2 = Z[v[2]];
            const int64_t area2 = ras_edge(x0, y0, x1, y1, x2, y2);
            if (area2 <= 0) continue;
            ++drawn;
            const int o12 = ras_owns(x1, y1, x2, y2), o20 = ras_owns(x2, y2, x0, y0), o01 = ras_owns(x0, y0, x1, y1);
            const float inv = 1.0f / (float)area2;
            const int64_t xmin = x0 < x1 ? (x0 < x2 ? x0 : x2) : (x1 < x2 ? x1 : x2);
            const int64_t xmax = x0 > x1 ? (x0 > x2 ? x0 : x2) : (x1 > x2 ? x1 : x2);
            const int64_t ymin = y0 < y1 ? (y0 < y2 ? y0 : y2) : (y1 < y2 ? y1 : y2);
            const int64_t ymax = y0 > y1 ? (y0 > y2 ? y0 : y2) : (y1 > y2 ? y1 : y2);
            int64_t px0 = -ras_floor256(-(xmin - 128)), px1 = ras_floor256(xmax - 128);
            int64_t py0 = -ras_floor256(-(ymin - 128)), py1 = ras_floor256(ymax - 128);
            px0 = px0 < 0 ? 0 : px0;
            py0 = py0 < 0 ? 0 : py0;
            px1 = px1 > (int64_t)width - 1 ? (int64_t)width - 1 : px1;
            py1 = py1 > (int64_t)height - 1 ? (int64_t)height - 1 : py1;
            for (int64_t py = py0; py <= py1; ++py)
                for (int64_t px = px0; px <= px1; ++px) {
                    const int64_t cx = px * 256 + 128, cy = py * 256 + 128;
                    const int64_t w0 = ras_edge(x1, y1, x2, y2, cx, cy), w1 = ras_edge(x2, y2, x0, y0, cx, cy),
                                  w2 = ras_edge(x0, y0, x1, y1, cx, cy);
                    if (!((w0 > 0 || (w0 == 0 && o12)) && (w1 > 0 || (w1 == 0 && o20)) && (w2 > 0 || (w2 == 0 && o01))))
                        continue;
                    float z = z0 + ((float)w1 * (z1 - z0) + (float)w2 * (z2 - z0)) * inv;
                    if (!(z > 0.0f)) z = 0.0f;
                    if (z > 1.0f) z = 1.0f;
                    ++frags;
                    const size_t at = (size_t)py * width + (size_t)px;
                    if (z <= depth[at]) { depth[at] = z; win[at] = i; }   /* GL_LEQUAL in draw order */
                }
        }
    }
    const uint32_t stride = stride_bytes / 4u;
    for (uint32_t y = 0; y < height; ++y)
        for (uint32_t x = 0; x < width; ++x) {
            const int64_t tri = win[(size_t)y * width + x];
            uint32_t out = 0u;
            if (tri >= 0) {
                const int32_t mi = d->tri_material ? d->tri_material[tri] : -1;
                V3 c;
                if (mi >= 0 && (uint32_t)mi < d->n_materials) {   /* glm::max(x, y) = x < y ? y : x */
                    const MrtMaterial *mt = &d->materials[mi];
                    c = vld(mt->kd);
                    c = v3(mt->ks[0] < c.x ? c.x : mt->ks[0], mt->ks[1] < c.y ? c.y : mt->ks[1], mt->ks[2] < c.z ? c.z : mt->ks[2]);
                    c = v3(mt->kt[0] < c.x ? c.x : mt->kt[0], mt->kt[1] < c.y ? c.y : mt->kt[1], mt->kt[2] < c.z ? c.z : mt->kt[2]);
                    c = v3(mt->le[0] < c.x ? c.x : mt->le[0], mt->le[1] < c.y ? c.y : mt->le[1], mt->le[2] < c.z ? c.z : mt->le[2]);
                } else if (d->tri_colors) {
                    const float *k3 = d->tri_colors + 9 * (size_t)tri;
                    c = v3(((k3[0] + k3[3]) + k3[6]) / 3.0f, ((k3[1] + k3[4]) + k3[7]) / 3.0f, ((k3[2] + k3[5]) + k3[8]) / 3.0f);
                } else {
                    c = v3(0.0f, 0.0f, 0.0f);
                }
                out = ras_unorm8(c.x) | (ras_unorm8(c.y) << 8) | (ras_unorm8(c.z) << 16) | (255u << 24);
            }
            bitmap[(size_t)(height - 1 - y) * stride + x] = out;
        }
    free(depth);
    free(win);
    if (counts) { counts[0] = drawn; counts[1] = frags; }
    return 0;
}
