/*
 * ffo.h — the CPU oracle: a plain-C restatement of the reference's hot-path
 * arithmetic (JakeKurtz/Firefly, CUDA-RayTracer/).  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this code, and only as the checker or the timed CPU baseline.  The
 * product (firefly_b200/) never calls it.
 *
 * Parity pins: tests/golden/ holds vectors produced by the reference's own
 * routines compiled for the host (oracle/_ref, recipe in oracle/Makefile);
 * tests/test_oracle_golden.py checks every function here against them.
 *
 * Build with -ffp-contract=off: every float expression is evaluated in the
 * reference's operand order with one rounding per operation, as the
 * reference's host build does (x86-64 SSE, no FMA).
 */
#ifndef FFO_H
#define FFO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- ray/triangle (dTriangle.cu:34-138) ---- */
/* dTriangle::intersect with TEST_CULL (dTriangle.cu:34-61): returns 1 on a
 * front-face hit and writes t, u, v; leaves them untouched on early exits. */
int ffo_intersect_cull(const float* v0, const float* v1, const float* v2,
                       const float* o, const float* d, float* t, float* u, float* v);
/* Two-sided closest-hit test (no reference counterpart): a front face is
 * ffo_intersect_cull; a back face passes the mirror image of it (negated
 * determinant and numerators) and sets *back. */
int ffo_intersect_two_sided(const float* v0, const float* v1, const float* v2,
                            const float* o, const float* d, float* t, float* u, float* v, int* back);
/* dTriangle::shadow_hit (dTriangle.cu:110-138): two-sided, u/v in double. */
int ffo_shadow_hit(const float* v0, const float* v1, const float* v2,
                   const float* o, const float* d, float* t);
/* The same three tests on v0 and the edges e1 = v1 - v0, e2 = v2 - v0 as the
 * reference rounds them (the device BVH stores the edges). */
int ffo_intersect_cull_e(const float* v0, const float* e1, const float* e2,
                         const float* o, const float* d, float* t, float* u, float* v);
int ffo_intersect_two_sided_e(const float* v0, const float* e1, const float* e2,
                              const float* o, const float* d, float* t, float* u, float* v, int* back);
int ffo_shadow_hit_e(const float* v0, const float* e1, const float* e2,
                     const float* o, const float* d, float* t);

/* Brute-force ray queries over a triangle soup (tris: n_tris x 9 floats,
 * v0 v1 v2).  rays: n x 8 floats (o, tmin, d, tmax) as ff_ray.  hits: n x 4
 * words (t, u, v as float bits, prim as int32).  any != 0 selects the any-hit
 * query.  Work is split over nthreads POSIX threads. */
void ffo_trace_brute(const float* tris, int64_t n_tris, const float* rays, int64_t n,
                     void* hits, int any, int nthreads);
/* The same with two_sided != 0 for two-sided closest hits (prim = -2 - id on
 * a back face). */
void ffo_trace_brute2(const float* tris, int64_t n_tris, const float* rays, int64_t n,
                      void* hits, int any, int two_sided, int nthreads);

/* The same queries over a CPU hierarchy (ffo_bvh.c), for large ray sets and
 * meshes: identical closest-hit answers (t, u, v, prim); any-hit reports
 * some occluder (prim >= 0) or -1, as ff_trace does. */
typedef struct ffo_bvh ffo_bvh;
ffo_bvh* ffo_bvh_build(const float* tris, int64_t n_tris);   /* keeps a pointer to tris */
void ffo_bvh_free(ffo_bvh* b);
void ffo_bvh_trace(const ffo_bvh* b, const float* rays, int64_t n, void* hits, int any, int two_sided,
                   int nthreads);

/* The device's own traversal restated (ffo_bvh8.c): the 8-wide quantised BVH
 * that ff_scene_read_bvh returns (nodes: num_nodes x 80-byte FFNode8, tris:
 * num_tris x 48-byte FFTri in leaf order) walked exactly as ff_traverse_step
 * walks it, with the same box arithmetic, child order, stack and triangle
 * tests.  hits as ffo_trace_brute2 (two_sided: a ray with the sign bit of tmin
 * set takes back faces, as the device's two-sided launches mark them);
 * counts[0] += node records fetched, counts[1] += triangles tested (ff_trace_count).
 * Returns the number of rays whose traversal overflowed its stack or step bound. */
int64_t ffo_bvh8_trace(const void* nodes, uint32_t num_nodes, const void* tris, uint32_t num_tris,
                       const float* rays, int64_t n, void* hits, int any, int two_sided,
                       uint64_t* counts, int nthreads);

/* ---- sampler (dRandom.cu:10-27) ---- */
uint32_t ffo_wang_hash(uint32_t s);
/* The seeded replacement of the reference's clock-seeded random():
 * wang_hash(key ^ wang_hash(dim)) * 2^-32 rounded to float (may be 1.0f,
 * as the reference's conversion may). */
float ffo_rand(uint32_t key, uint32_t dim);
/* Per-(pixel, sample) stream key. */
uint32_t ffo_path_key(uint32_t seed, uint32_t pixel, uint32_t sample);

/* ---- CPU render (restated wavefront stages, ffo_render.c) ---- */
typedef struct {
    float base_color[3];
    float fresnel[3];
    float roughness;
    float metallic;
    int32_t kind;          /* 0 mix (wf_mat_mix), 1 diffuse (wf_mat_diffuse), 2 conductor (wf_mat_cook),
                              3 rough dielectric, 4 diffuse under a GGX coat (no reference counterparts) */
    int32_t base_color_tex;  /* -1 = none */
    int32_t roughness_tex;   /* -1 = none */
    int32_t metallic_tex;    /* -1 = none */
    int32_t metallic_roughness_tex; /* -1 = none (glTF packing: roughness y, metallic z) */
    int32_t normal_tex;      /* -1 = none (tangent space) */
    float ior;               /* kinds 3 (dielectric) and 4 (coat); <= 0 means 1.5 */
} ffo_material;

typedef struct {
    const float* rgb;      /* height x width x 3 */
    int32_t width, height;
} ffo_texture;

typedef struct {
    float p0[3], a[3], b[3], normal[3];
    float emissive[3];
    float radiance;
} ffo_area_light;

/* dDirectionalLight (dDirectionalLight.cu:5-57): direction toward the light
 * (normalised by ffo_render in double), radiance * emissive, pdf 1, delta. */
typedef struct ffo_dir_light {
    float direction[3];
    float emissive[3];
    float radiance;
    float pad;
} ffo_dir_light;

typedef struct {
    const float* tris;          /* num_tris x 9: v0 v1 v2 */
    const float* normals;       /* num_tris x 9: vertex normals n0 n1 n2 */
    const uint32_t* material_ids;
    int32_t num_tris;
    const float* texcoords;     /* num_tris x 6: uv0 uv1 uv2, or NULL */
    const ffo_texture* textures;
    int32_t num_textures;
    const ffo_material* materials;
    int32_t num_materials;
    const ffo_area_light* area_lights;
    int32_t num_area_lights;
    const float* env_rgb;       /* env_h x env_w x 3, or NULL (constant env_color) */
    int32_t env_w, env_h;
    float env_color[3];
    float cam_inv[16];          /* Matrix4x4 m[i][j] at 4*i + j */
    float cam_lens_radius, cam_focal, cam_jitter;
    int32_t width, height, spp, sample_offset, max_depth, rr_depth;
    uint32_t seed;
    int32_t mode;               /* 0 parity, 1 corrected */
    int32_t light;              /* -1 environment, k area light k */
    float shadow_offset;
    int32_t threads;
    /* light: -1 env, 0..A-1 area, A..A+D-1 directional, -2 one light per
     * vertex chosen uniformly among all (corrected mode) */
    const ffo_dir_light* dir_lights;
    int32_t num_dir_lights;
    /* per-triangle vertex tangents and bitangents (num_tris x 9 each) for
     * normal textures, or NULL */
    const float* tangents;
    const float* bitangents;
} ffo_render_desc;

/* Renders every pixel's spp samples; out_rgb (width*height*3 doubles) gets
 * the per-pixel radiance sums.  stats[0..1] = extension and shadow rays.
 * Returns 0, or 1 for an invalid light selection. */
int ffo_render(const ffo_render_desc* d, double* out_rgb, uint64_t* stats);

/* Material texture reads (get_albedo / get_roughness / get_metallic /
 * get_normal, dMaterial.cu:10-88) at one intersection: isect11 = texcoord[2],
 * normal[3], tangent[3], bitangent[3]; out8 = albedo[3], roughness, metallic,
 * normal[3]. */
void ffo_probe_surface(const ffo_material* mm, const ffo_texture* textures, const float* isect11, float* out8);

/* Environment tables of kernel.cu:65-149 (marginal[h], cond[h*w], pdf[h*w]). */
void ffo_env_build(const float* rgb, int w, int h, double* marginal, double* cond, float* pdf, double* denom);

#ifdef __cplusplus
}
#endif

#endif
