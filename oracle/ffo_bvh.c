/*
 * ffo_bvh.c — the oracle's ray queries over a CPU bounding-volume hierarchy,
 * for ray sets too large for ffo_trace_brute (the 4 x 16.8M rays of the
 * trace micro-benchmark, the 1.3M-triangle at-scale mesh).  TEST
 * INFRASTRUCTURE ONLY (see ffo.h).  Compile with -ffp-contract=off.
 *
 * The answers are exactly ffo_trace_brute's: every triangle is decided by
 * the same restated tests (ffo_intersect_cull / ffo_intersect_two_sided /
 * ffo_shadow_hit, which follow CUDA-RayTracer/dTriangle.cu:34-138), the
 * closest hit is the smallest t with ties to the lowest index, and the
 * hierarchy only skips triangles that cannot be hit: boxes are padded by
 * 1e-5 of the scene's extent and the ray's interval is widened by 1e-4 of
 * the current best distance (plus 1e-4 of the extent), both far beyond the
 * float rounding by which the reference's tests can accept a point outside
 * the exact triangle, and the slab tests run in double.  Binary hierarchy,
 * median split of the centroids on the widest axis, leaves of at most 4
 * triangles, the near child first; an explicit stack; POSIX threads over
 * the rays.
 */
#include "ffo.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define BVH_LEAF 4
#define BVH_STACK 128

typedef struct {
    double lo[3], hi[3];
    int32_t a, b;          /* inner: children a (smaller centroids), b; leaf: first index a, count -b */
    int32_t axis;          /* inner: split axis */
} bnode;

struct ffo_bvh {
    bnode* nodes;
    int32_t* idx;
    int64_t n_nodes;
    const float* tris;
    int64_t n_tris;
    double pad, t_pad;
};

static float* g_cent;   /* centroid of the triangle being partitioned (build only, one thread) */

static void tri_bounds(const float* t, double lo[3], double hi[3])
{
    for (int k = 0; k < 3; ++k) {
        double a = t[k], b = t[3 + k], c = t[6 + k];
        double mn = a < b ? a : b, mx = a > b ? a : b;
        lo[k] = mn < c ? mn : c;
        hi[k] = mx > c ? mx : c;
    }
}

/* k-th smallest centroid on axis `ax` moved to position k (quickselect). */
static void select_k(int32_t* idx, int64_t n, int64_t k, int ax)
{
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        float pivot = g_cent[3 * (int64_t)idx[(lo + hi) / 2] + ax];
        int64_t i = lo, j = hi;
        while (i <= j) {
            while (g_cent[3 * (int64_t)idx[i] + ax] < pivot) ++i;
            while (g_cent[3 * (int64_t)idx[j] + ax] > pivot) --j;
            if (i <= j) {
                int32_t t = idx[i];
                idx[i] = idx[j];
                idx[j] = t;
                ++i;
                --j;
            }
        }
        if (k <= j) hi = j;
        else if (k >= i) lo = i;
        else return;
    }
}

static int64_t build_rec(struct ffo_bvh* b, int64_t first, int64_t count)
{
    int64_t me = b->n_nodes++;
    bnode* nd = &b->nodes[me];
    for (int k = 0; k < 3; ++k) {
        nd->lo[k] = INFINITY;
        nd->hi[k] = -INFINITY;
    }
    double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = first; i < first + count; ++i) {
        double lo[3], hi[3];
        const int64_t t = b->idx[i];
        tri_bounds(b->tris + 9 * t, lo, hi);
        for (int k = 0; k < 3; ++k) {
            if (lo[k] < nd->lo[k]) nd->lo[k] = lo[k];
            if (hi[k] > nd->hi[k]) nd->hi[k] = hi[k];
            double c = g_cent[3 * t + k];
            if (c < clo[k]) clo[k] = c;
            if (c > chi[k]) chi[k] = c;
        }
    }
    for (int k = 0; k < 3; ++k) {
        nd->lo[k] -= b->pad;
        nd->hi[k] += b->pad;
    }
    if (count <= BVH_LEAF) {
        nd->a = (int32_t)first;
        nd->b = -(int32_t)count;
        return me;
    }
    int ax = 0;
    for (int k = 1; k < 3; ++k)
        if (chi[k] - clo[k] > chi[ax] - clo[ax]) ax = k;
    int64_t half = count / 2;
    select_k(b->idx + first, count, half, ax);
    int64_t l = build_rec(b, first, half);
    int64_t r = build_rec(b, first + half, count - half);
    b->nodes[me].a = (int32_t)l;
    b->nodes[me].b = (int32_t)r;
    b->nodes[me].axis = ax;
    return me;
}

ffo_bvh* ffo_bvh_build(const float* tris, int64_t n_tris)
{
    struct ffo_bvh* b = (struct ffo_bvh*)calloc(1, sizeof(*b));
    if (!b) return NULL;
    b->tris = tris;
    b->n_tris = n_tris;
    if (n_tris == 0) return b;
    b->nodes = (bnode*)malloc(sizeof(bnode) * (size_t)(2 * n_tris));
    b->idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)n_tris);
    g_cent = (float*)malloc(sizeof(float) * 3 * (size_t)n_tris);
    if (!b->nodes || !b->idx || !g_cent) {
        free(g_cent);
        ffo_bvh_free(b);
        return NULL;
    }
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t t = 0; t < n_tris; ++t) {
        b->idx[t] = (int32_t)t;
        const float* p = tris + 9 * t;
        for (int k = 0; k < 3; ++k) {
            g_cent[3 * t + k] = (p[k] + p[3 + k] + p[6 + k]) / 3.0f;
            for (int v = 0; v < 3; ++v) {
                if (p[3 * v + k] < lo[k]) lo[k] = p[3 * v + k];
                if (p[3 * v + k] > hi[k]) hi[k] = p[3 * v + k];
            }
        }
    }
    double ext = 0.0;
    for (int k = 0; k < 3; ++k) {
        double e = hi[k] - lo[k];
        double m = fabs(lo[k]) > fabs(hi[k]) ? fabs(lo[k]) : fabs(hi[k]);
        if (e > ext) ext = e;
        if (m > ext) ext = m;
    }
    b->pad = 1e-5 * ext + 1e-30;
    b->t_pad = 1e-4 * ext + 1e-30;
    build_rec(b, 0, n_tris);
    free(g_cent);
    g_cent = NULL;
    return b;
}

void ffo_bvh_free(ffo_bvh* b)
{
    if (!b) return;
    free(b->nodes);
    free(b->idx);
    free(b);
}

/* Does the ray (o, d) meet the padded box for some t in [t0, t1]? */
static int box_hit(const bnode* nd, const double o[3], const double d[3], double t0, double t1)
{
    for (int k = 0; k < 3; ++k) {
        if (d[k] == 0.0) {
            if (o[k] < nd->lo[k] || o[k] > nd->hi[k]) return 0;
            continue;
        }
        double a = (nd->lo[k] - o[k]) / d[k], c = (nd->hi[k] - o[k]) / d[k];
        if (a > c) {
            double s = a;
            a = c;
            c = s;
        }
        if (a > t0) t0 = a;
        if (c < t1) t1 = c;
        if (t0 > t1) return 0;
    }
    return 1;
}

typedef struct {
    const struct ffo_bvh* b;
    const float* rays;
    int64_t begin, end;
    uint32_t* hits;
    int any, two_sided;
} bjob_t;

static void* run_bjob(void* arg)
{
    bjob_t* j = (bjob_t*)arg;
    const struct ffo_bvh* b = j->b;
    int32_t stack[BVH_STACK];
    for (int64_t r = j->begin; r < j->end; ++r) {
        const float* ray = j->rays + 8 * r;
        const float of[3] = {ray[0], ray[1], ray[2]};
        const float df[3] = {ray[4], ray[5], ray[6]};
        const double o[3] = {ray[0], ray[1], ray[2]}, d[3] = {ray[4], ray[5], ray[6]};
        const float tmin = ray[3], tmax = ray[7];
        float best_t = j->any ? tmax : (tmax < 1e32f ? tmax : 1e32f);
        float best_u = 0.f, best_v = 0.f;
        int32_t best = -1, best_id = -1;
        int sp = 0;
        if (b->n_tris) stack[sp++] = 0;
        int done = 0;
        while (sp > 0 && !done) {
            const bnode* nd = &b->nodes[stack[--sp]];
            double lim = (double)best_t;
            if (!(lim < 1e300)) lim = 1e300;   /* tmax may be inf */
            if (!box_hit(nd, o, d, (double)tmin - b->t_pad, lim + 1e-4 * fabs(lim) + b->t_pad)) continue;
            if (nd->b <= 0) {
                for (int32_t q = nd->a; q < nd->a - nd->b; ++q) {
                    const int32_t id = b->idx[q];
                    const float* tri = b->tris + 9 * (int64_t)id;
                    float t, u, v;
                    if (j->any) {
                        if (ffo_shadow_hit(tri, tri + 3, tri + 6, of, df, &t) && t >= tmin && t < tmax) {
                            best = id;
                            best_t = t;
                            done = 1;
                            break;
                        }
                        continue;
                    }
                    int back = 0;
                    int ok = j->two_sided ? ffo_intersect_two_sided(tri, tri + 3, tri + 6, of, df, &t, &u, &v, &back)
                                          : ffo_intersect_cull(tri, tri + 3, tri + 6, of, df, &t, &u, &v);
                    if (!ok || t < 0 || !(t >= tmin)) continue;
                    if (t < best_t || (t == best_t && best_id >= 0 && id < best_id)) {
                        best_t = t;
                        best_u = u;
                        best_v = v;
                        best_id = id;
                        best = back ? -2 - id : id;
                    }
                }
            } else {
                if (sp + 2 > BVH_STACK) {   /* deeper than any median-split tree of 2^31 triangles */
                    best = -1;
                    break;
                }
                /* the child on the ray's near side first */
                const int near_a = d[nd->axis] >= 0.0;
                stack[sp++] = near_a ? nd->b : nd->a;
                stack[sp++] = near_a ? nd->a : nd->b;
            }
        }
        uint32_t* h = j->hits + 4 * r;
        float out[3];
        if (best == -1) {
            out[0] = j->any ? tmax : (tmax < 1e32f ? tmax : 1e32f);
            out[1] = out[2] = 0.f;
        } else {
            out[0] = best_t;
            out[1] = j->any ? 0.f : best_u;
            out[2] = j->any ? 0.f : best_v;
        }
        memcpy(h, out, 12);
        memcpy(h + 3, &best, 4);
    }
    return NULL;
}

void ffo_bvh_trace(const ffo_bvh* b, const float* rays, int64_t n, void* hits, int any, int two_sided, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    bjob_t jobs[256];
    int64_t chunk = (n + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
        jobs[k].b = b;
        jobs[k].rays = rays;
        jobs[k].begin = k * chunk < n ? k * chunk : n;
        jobs[k].end = (k + 1) * chunk < n ? (k + 1) * chunk : n;
        jobs[k].hits = (uint32_t*)hits;
        jobs[k].any = any;
        jobs[k].two_sided = two_sided;
        if (pthread_create(&th[k], NULL, run_bjob, &jobs[k]) != 0) {
            run_bjob(&jobs[k]);
            th[k] = 0;
        }
    }
    for (int k = 0; k < nthreads; ++k)
        if (th[k]) pthread_join(th[k], NULL);
}
