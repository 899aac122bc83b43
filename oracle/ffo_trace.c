/*
 * ffo_trace.c — CPU restatement of the reference's ray/triangle tests and a
 * brute-force closest-hit / any-hit query.  TEST INFRASTRUCTURE ONLY (see
 * ffo.h).  Compile with -ffp-contract=off.
 *
 * Follows CUDA-RayTracer/dTriangle.cu:
 *   dTriangle::intersect   :34-61  (TEST_CULL defined at :5)
 *   dTriangle::hit         :89-108 (rejects t < 0)
 *   dTriangle::shadow_hit  :110-138
 *   intersect()            :140-213 (accepts t < tmin, tmin starts at K_HUGE)
 *   intersect_shadows()    :215-259 (accepts t < tmin, early exit)
 * and the vector helpers of CUDA-RayTracer/dMath.cuh (dot :1222, cross :1411,
 * K_EPSILON = 1e-6f :78, K_HUGE = 1e32f :80).
 */
#include "ffo.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define FFO_K_EPSILON 1e-6f
#define FFO_K_HUGE 1e32f

typedef struct { float x, y, z; } v3;

static inline v3 mk(const float* p) { v3 r = {p[0], p[1], p[2]}; return r; }
static inline v3 sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
/* dMath.cuh:1222: a.x*b.x + a.y*b.y + a.z*b.z, left to right. */
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* dMath.cuh:1411. */
static inline v3 cross(v3 a, v3 b)
{
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}

/* The tests below on the vertex v0 and the edges e1 = v1 - v0, e2 = v2 - v0
 * as the reference rounds them (dTriangle.cu:35-36); the *_e forms take the
 * edges directly (the device BVH stores them, ffo_bvh8.c). */
int ffo_intersect_cull_e(const float* p0, const float* pe1, const float* pe2,
                         const float* po, const float* pd, float* t, float* u, float* v)
{
    v3 v0 = mk(p0), e1 = mk(pe1), e2 = mk(pe2), o = mk(po), d = mk(pd);
    v3 pvec = cross(d, e2);
    double det = dot(e1, pvec);             /* float dot widened to double */
    if (det < FFO_K_EPSILON) return 0;      /* K_EPSILON is a float constant */
    v3 tvec = sub(o, v0);
    float uu = dot(tvec, pvec);
    *u = uu;
    if (uu < 0.0 || uu > det) return 0;
    v3 qvec = cross(tvec, e1);
    float vv = dot(d, qvec);
    *v = vv;
    if (vv < 0.0 || uu + vv > det) return 0;   /* float add, double compare */
    float tt = dot(e2, qvec);
    double inv_det = 1.0 / det;
    *t = (float)(tt * inv_det);
    *u = (float)(uu * inv_det);
    *v = (float)(vv * inv_det);
    return 1;
}

int ffo_intersect_cull(const float* p0, const float* p1, const float* p2,
                       const float* po, const float* pd, float* t, float* u, float* v)
{
    v3 v0 = mk(p0), v1 = mk(p1), v2 = mk(p2);
    v3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    return ffo_intersect_cull_e(p0, &e1.x, &e2.x, po, pd, t, u, v);
}

/* Two-sided closest-hit test (no reference counterpart: the reference only
 * culls, dTriangle.cu:5,41).  A front face (det >= K_EPSILON) is exactly
 * ffo_intersect_cull; a back face (det <= -K_EPSILON) runs the same test on
 * the negated determinant and numerators (negation is exact), the mirror
 * image of the culling test.  *back reports which.  The product restates it
 * in ff_test_tri_closest<TWO> (firefly_b200/csrc/ff_trace.cuh). */
int ffo_intersect_two_sided_e(const float* p0, const float* pe1, const float* pe2,
                              const float* po, const float* pd, float* t, float* u, float* v, int* back)
{
    v3 v0 = mk(p0), e1 = mk(pe1), e2 = mk(pe2), o = mk(po), d = mk(pd);
    v3 pvec = cross(d, e2);
    float detf = dot(e1, pvec);
    float sg = 1.f;
    *back = 0;
    if (detf < FFO_K_EPSILON) {
        if (!(detf <= -FFO_K_EPSILON)) return 0;
        sg = -1.f;
        *back = 1;
    }
    double det = (double)(sg * detf);
    v3 tvec = sub(o, v0);
    float uu = sg * dot(tvec, pvec);
    if (uu < 0.0 || uu > det) return 0;
    v3 qvec = cross(tvec, e1);
    float vv = sg * dot(d, qvec);
    if (vv < 0.0 || uu + vv > det) return 0;
    float tt = sg * dot(e2, qvec);
    double inv_det = 1.0 / det;
    *t = (float)(tt * inv_det);
    *u = (float)(uu * inv_det);
    *v = (float)(vv * inv_det);
    return 1;
}

int ffo_intersect_two_sided(const float* p0, const float* p1, const float* p2,
                            const float* po, const float* pd, float* t, float* u, float* v, int* back)
{
    v3 v0 = mk(p0), v1 = mk(p1), v2 = mk(p2);
    v3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    return ffo_intersect_two_sided_e(p0, &e1.x, &e2.x, po, pd, t, u, v, back);
}

int ffo_shadow_hit_e(const float* p0, const float* pe1, const float* pe2,
                     const float* po, const float* pd, float* t)
{
    v3 v0 = mk(p0), e1 = mk(pe1), e2 = mk(pe2), o = mk(po), d = mk(pd);
    v3 pvec = cross(d, e2);
    double det = dot(e1, pvec);
    if (det > -FFO_K_EPSILON && det < FFO_K_EPSILON) return 0;
    double inv_det = 1.0 / det;
    v3 tvec = sub(o, v0);
    double u = dot(tvec, pvec) * inv_det;
    if (u < 0.0 || u > 1.0) return 0;
    v3 qvec = cross(tvec, e1);
    double v = dot(d, qvec) * inv_det;
    if (v < 0.0 || u + v > 1.0) return 0;
    float tt = (float)(dot(e2, qvec) * inv_det);
    *t = tt;
    if (tt < 0) return 0;
    return 1;
}

int ffo_shadow_hit(const float* p0, const float* p1, const float* p2,
                   const float* po, const float* pd, float* t)
{
    v3 v0 = mk(p0), v1 = mk(p1), v2 = mk(p2);
    v3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    return ffo_shadow_hit_e(p0, &e1.x, &e2.x, po, pd, t);
}

typedef struct {
    const float* tris;
    int64_t n_tris;
    const float* rays;
    int64_t begin, end;
    uint32_t* hits;
    int any;
    int two_sided;
} job_t;

static void* run_job(void* arg)
{
    job_t* j = (job_t*)arg;
    for (int64_t r = j->begin; r < j->end; ++r) {
        const float* ray = j->rays + 8 * r;
        const float o[3] = {ray[0], ray[1], ray[2]};
        const float d[3] = {ray[4], ray[5], ray[6]};
        const float tmin = ray[3];
        const float tmax = ray[7];
        float best_t = tmax < FFO_K_HUGE ? tmax : FFO_K_HUGE;
        float best_u = 0.f, best_v = 0.f;
        int32_t best = -1;
        for (int64_t i = 0; i < j->n_tris; ++i) {
            const float* tri = j->tris + 9 * i;
            float t, u, v;
            if (j->any) {
                if (ffo_shadow_hit(tri, tri + 3, tri + 6, o, d, &t) && t >= tmin && t < tmax) {
                    best = (int32_t)i;
                    best_t = t;
                    break;
                }
            } else if (j->two_sided) {
                /* strict < over increasing ids: ties go to the lowest id; a
                 * back face is reported as -2 - id */
                int back = 0;
                if (ffo_intersect_two_sided(tri, tri + 3, tri + 6, o, d, &t, &u, &v, &back) &&
                    !(t < 0) && t >= tmin && t < best_t) {
                    best = back ? -2 - (int32_t)i : (int32_t)i;
                    best_t = t;
                    best_u = u;
                    best_v = v;
                }
            } else {
                /* strict < over increasing ids: ties go to the lowest id */
                if (ffo_intersect_cull(tri, tri + 3, tri + 6, o, d, &t, &u, &v) &&
                    !(t < 0) && t >= tmin && t < best_t) {
                    best = (int32_t)i;
                    best_t = t;
                    best_u = u;
                    best_v = v;
                }
            }
        }
        uint32_t* h = j->hits + 4 * r;
        float out[3];
        if (best == -1) {
            out[0] = j->any ? tmax : (tmax < FFO_K_HUGE ? tmax : FFO_K_HUGE);
            out[1] = 0.f;
            out[2] = 0.f;
        } else {
            out[0] = best_t;
            out[1] = best_u;
            out[2] = best_v;
        }
        memcpy(h, out, 12);
        memcpy(h + 3, &best, 4);
    }
    return NULL;
}

void ffo_trace_brute(const float* tris, int64_t n_tris, const float* rays, int64_t n,
                     void* hits, int any, int nthreads)
{
    ffo_trace_brute2(tris, n_tris, rays, n, hits, any, 0, nthreads);
}

void ffo_trace_brute2(const float* tris, int64_t n_tris, const float* rays, int64_t n,
                      void* hits, int any, int two_sided, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    job_t jobs[256];
    int64_t chunk = (n + nthreads - 1) / nthreads;
    int started = 0;
    for (int k = 0; k < nthreads; ++k) {
        jobs[k].tris = tris;
        jobs[k].n_tris = n_tris;
        jobs[k].rays = rays;
        jobs[k].begin = k * chunk < n ? k * chunk : n;
        jobs[k].end = (k + 1) * chunk < n ? (k + 1) * chunk : n;
        jobs[k].hits = (uint32_t*)hits;
        jobs[k].any = any;
        jobs[k].two_sided = two_sided;
        if (pthread_create(&th[k], NULL, run_job, &jobs[k]) == 0) {
            started |= 0;
        } else {
            run_job(&jobs[k]);
            th[k] = 0;
        }
    }
    for (int k = 0; k < nthreads; ++k)
        if (th[k]) pthread_join(th[k], NULL);
    (void)started;
}

/* dRandom.cu:10-18. */
uint32_t ffo_wang_hash(uint32_t s)
{
    s = (s ^ 61u) ^ (s >> 16);
    s *= 9u;
    s = s ^ (s >> 4);
    s *= 0x27d4eb2du;
    s = s ^ (s >> 15);
    return s;
}

/* dRandom.cu:26: wang_hash(seed) * (1.0 / 4294967296.0) returned as float. */
float ffo_rand(uint32_t key, uint32_t dim)
{
    uint32_t h = ffo_wang_hash(key ^ ffo_wang_hash(dim));
    return (float)((double)h * (1.0 / 4294967296.0));
}

uint32_t ffo_path_key(uint32_t seed, uint32_t pixel, uint32_t sample)
{
    return ffo_wang_hash(ffo_wang_hash(ffo_wang_hash(seed) ^ pixel) + sample);
}
