/*
 * ffo_bvh8.c — the device traversal restated on the CPU, over the 8-wide
 * quantised BVH the device built (read back with ff_scene_read_bvh).  TEST
 * INFRASTRUCTURE ONLY (see ffo.h).  Compile with -ffp-contract=off: every
 * fused multiply-add below is an explicit fmaf, as the device code writes it.
 *
 * Follows firefly_b200/csrc/ff_trace.cuh step by step:
 *   ff_ray_setup        safe reciprocal of the direction (1 / +-1e-20 for
 *                       components below 1e-20), octant, tmax clamped to
 *                       K_HUGE for closest hits;
 *   ff_intersect_node   slab distances fmaf(plane byte, 2^e / d, (p - o) / d)
 *                       per axis, near and far planes chosen by the sign of
 *                       1 / d, three-input max / min, widening by 2^-12 of
 *                       |t| (fmaf), entry test max(tn, tmin) <= min(tf, tb);
 *                       hit internal children set bit 24 + (slot ^ octant),
 *                       hit leaves add their unary triangle mask;
 *   ff_traverse_step    next child = highest hit bit, slot = bit ^ octant,
 *                       child index = child_base + internal children in lower
 *                       slots; the rest of the group is pushed; then the
 *                       exposed triangles in bit order; then a pop;
 * and the triangle tests of ffo_trace.c (the reference's, which the device's
 * tests match bit for bit) with the device's acceptance rules: closest hits
 * take t >= tmin and t < best, or t == best with a lower original index; any
 * hit stops at the first t in [tmin, tmax).
 */
#include "ffo.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define K_HUGE 1e32f
#define BOX_WIDEN 2.44140625e-4f   /* 2^-12 */
#define MAX_STACK 64
#define BACK_FACE 0x80000000u

typedef struct {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
} node8_t;

typedef struct {
    float a[4], b[4], c[4];   /* v0 + original index bits, e1, e2 */
} tri48_t;

typedef struct {
    float o[3], d[3], inv[3];
    float tmin, tmax, u, v;
    uint32_t prim, oct_inv;
} ray_t;

typedef struct {
    uint32_t x, y;
} group_t;

static float safe_inv(float x)
{
    const float tiny = 1e-20f;
    return 1.0f / (fabsf(x) > tiny ? x : copysignf(tiny, x));
}

static float pow2_of_byte(uint8_t e)
{
    const uint32_t bits = (uint32_t)e << 23;
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static float max3(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }
static float min3(float a, float b, float c) { return fminf(fminf(a, b), c); }

static void intersect_node(const node8_t* nd, const ray_t* r, group_t* node_group, group_t* tri_group)
{
    const float sx = pow2_of_byte(nd->ex), sy = pow2_of_byte(nd->ey), sz = pow2_of_byte(nd->ez);
    const float ax = sx * r->inv[0], ay = sy * r->inv[1], az = sz * r->inv[2];
    const float bx = (nd->px - r->o[0]) * r->inv[0], by = (nd->py - r->o[1]) * r->inv[1],
                bz = (nd->pz - r->o[2]) * r->inv[2];
    const uint8_t* nx = r->inv[0] >= 0.f ? nd->qlox : nd->qhix;
    const uint8_t* fx = r->inv[0] >= 0.f ? nd->qhix : nd->qlox;
    const uint8_t* ny = r->inv[1] >= 0.f ? nd->qloy : nd->qhiy;
    const uint8_t* fy = r->inv[1] >= 0.f ? nd->qhiy : nd->qloy;
    const uint8_t* nz = r->inv[2] >= 0.f ? nd->qloz : nd->qhiz;
    const uint8_t* fz = r->inv[2] >= 0.f ? nd->qhiz : nd->qloz;
    const float tb = fmaf(fabsf(r->tmax), BOX_WIDEN, r->tmax);
    uint32_t hits = 0, tmask = 0;
    for (int s = 0; s < 8; ++s) {
        float tn = max3(fmaf((float)nx[s], ax, bx), fmaf((float)ny[s], ay, by), fmaf((float)nz[s], az, bz));
        float tf = min3(fmaf((float)fx[s], ax, bx), fmaf((float)fy[s], ay, by), fmaf((float)fz[s], az, bz));
        tn = fmaf(-fabsf(tn), BOX_WIDEN, tn);
        tf = fmaf(fabsf(tf), BOX_WIDEN, tf);
        if (fmaxf(tn, r->tmin) <= fminf(tf, tb)) {
            const uint32_t meta = nd->meta[s];
            if ((nd->imask >> s) & 1u) hits |= 1u << (24 + (s ^ r->oct_inv));
            else tmask |= (meta >> 5) << (meta & 31u);
        }
    }
    node_group->x = nd->child_base;
    node_group->y = hits | nd->imask;
    tri_group->x = nd->tri_base;
    tri_group->y = tmask;
}

/* ff_test_tri_closest / ff_test_tri_any on the reference's tests. */
static void test_closest(const tri48_t* t, ray_t* r, int two)
{
    float tt, u, v;
    int back = 0;
    int ok;
    const int two_ray = two && signbit(r->tmin);
    if (two_ray) ok = ffo_intersect_two_sided_e(t->a, t->b, t->c, r->o, r->d, &tt, &u, &v, &back);
    else ok = ffo_intersect_cull_e(t->a, t->b, t->c, r->o, r->d, &tt, &u, &v);
    if (!ok) return;
    if (tt < 0.f || !(tt >= (two ? fabsf(r->tmin) : r->tmin))) return;
    uint32_t id;
    memcpy(&id, &t->a[3], 4);
    const uint32_t best = two ? (r->prim & ~BACK_FACE) : r->prim;
    if (tt < r->tmax || (tt == r->tmax && r->prim != 0xffffffffu && id < best)) {
        r->tmax = tt;
        r->prim = back ? (id | BACK_FACE) : id;
        r->u = u;
        r->v = v;
    }
}

static int test_any(const tri48_t* t, ray_t* r)
{
    float tt;
    if (!ffo_shadow_hit_e(t->a, t->b, t->c, r->o, r->d, &tt)) return 0;
    if (tt >= r->tmin && tt < r->tmax) {
        uint32_t id;
        memcpy(&id, &t->a[3], 4);
        r->prim = id;
        r->tmax = tt;
        return 1;
    }
    return 0;
}

typedef struct {
    const node8_t* nodes;
    uint32_t num_nodes;
    const tri48_t* tris;
    uint32_t num_tris;
    const float* rays;
    int64_t begin, end;
    uint32_t* hits;
    int any, two;
    uint64_t nodes_n, tris_n;
    int64_t errors;
} job8_t;

static void* run_job8(void* arg)
{
    job8_t* j = (job8_t*)arg;
    group_t stack[MAX_STACK];
    for (int64_t k = j->begin; k < j->end; ++k) {
        const float* ray = j->rays + 8 * k;
        ray_t r;
        for (int a = 0; a < 3; ++a) {
            r.o[a] = ray[a];
            r.d[a] = ray[4 + a];
            r.inv[a] = safe_inv(ray[4 + a]);
        }
        /* a two-sided launch (ff_trace with FF_TRACE_TWO_SIDED) marks every
         * ray: tmin = -max(tmin, 0), whose sign bit selects back faces */
        r.tmin = j->two ? -(ray[3] > 0.f ? ray[3] : 0.f) : ray[3];
        r.tmax = j->any ? ray[7] : fminf(ray[7], K_HUGE);
        r.u = r.v = 0.f;
        r.prim = 0xffffffffu;
        r.oct_inv = (r.d[0] < 0.f ? 0u : 1u) | (r.d[1] < 0.f ? 0u : 2u) | (r.d[2] < 0.f ? 0u : 4u);
        int sp = 0, overflow = 0;
        uint32_t steps = 0;
        group_t cur = {0u, (1u << 31) | (1u << (7u ^ r.oct_inv))};
        int done = j->num_nodes == 0;
        while (!done) {
            group_t tri_group = {0u, 0u};
            if (cur.y & 0xff000000u) {
                const uint32_t bit = 31u - (uint32_t)__builtin_clz(cur.y & 0xff000000u);
                cur.y &= ~(1u << bit);
                const uint32_t slot = (bit - 24u) ^ r.oct_inv;
                const uint32_t child = cur.x + (uint32_t)__builtin_popcount(cur.y & 0xffu & ((1u << slot) - 1u));
                if (cur.y & 0xff000000u) {
                    if (sp >= MAX_STACK) overflow = 1;
                    else stack[sp++] = cur;
                }
                if (child >= j->num_nodes) {
                    overflow = 1;
                    break;
                }
                ++j->nodes_n;
                intersect_node(&j->nodes[child], &r, &cur, &tri_group);
            }
            int hit_any = 0;
            while (tri_group.y) {
                const uint32_t i = (uint32_t)__builtin_ctz(tri_group.y);
                tri_group.y &= tri_group.y - 1u;
                if (tri_group.x + i >= j->num_tris) {
                    overflow = 1;
                    break;
                }
                ++j->tris_n;
                if (j->any) {
                    if (test_any(&j->tris[tri_group.x + i], &r)) {
                        hit_any = 1;
                        break;
                    }
                } else {
                    test_closest(&j->tris[tri_group.x + i], &r, j->two);
                }
            }
            if (hit_any || overflow) break;
            if (!(cur.y & 0xff000000u)) {
                if (sp == 0) break;
                cur = stack[--sp];
            }
            if (++steps > j->num_nodes + 2u) {
                overflow = 1;
                break;
            }
        }
        if (overflow) ++j->errors;
        uint32_t* h = j->hits + 4 * k;
        int32_t prim = -1;
        if (r.prim != 0xffffffffu) {
            const int32_t id = (int32_t)(r.prim & ~BACK_FACE);
            prim = (j->two && (r.prim & BACK_FACE)) ? -2 - id : id;
        }
        float out[3] = {r.tmax, r.u, r.v};
        memcpy(h, out, 12);
        memcpy(h + 3, &prim, 4);
    }
    return NULL;
}

int64_t ffo_bvh8_trace(const void* nodes, uint32_t num_nodes, const void* tris, uint32_t num_tris,
                       const float* rays, int64_t n, void* hits, int any, int two_sided,
                       uint64_t* counts, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    job8_t jobs[256];
    const int64_t chunk = (n + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
        job8_t* j = &jobs[k];
        j->nodes = (const node8_t*)nodes;
        j->num_nodes = num_nodes;
        j->tris = (const tri48_t*)tris;
        j->num_tris = num_tris;
        j->rays = rays;
        j->begin = k * chunk < n ? k * chunk : n;
        j->end = (k + 1) * chunk < n ? (k + 1) * chunk : n;
        j->hits = (uint32_t*)hits;
        j->any = any;
        j->two = two_sided && !any;
        j->nodes_n = j->tris_n = 0;
        j->errors = 0;
        if (pthread_create(&th[k], NULL, run_job8, j) != 0) {
            run_job8(j);
            th[k] = 0;
        }
    }
    int64_t errors = 0;
    for (int k = 0; k < nthreads; ++k) {
        if (th[k]) pthread_join(th[k], NULL);
        counts[0] += jobs[k].nodes_n;
        counts[1] += jobs[k].tris_n;
        errors += jobs[k].errors;
    }
    return errors;
}
