/*
 * firefly_b200.h — C ABI of the B200 (sm_100a) wavefront path tracer.
 *
 * The reference (JakeKurtz/Firefly, directory CUDA-RayTracer/) reaches its
 * device code through C++ free functions defined in kernel.cu and called from
 * the dScene and PathTracer classes.  This header is the replacement seam: plain
 * C types, plain pointers and sizes, status codes instead of exit()/abort().
 * Each entry point names the reference interface it replaces.
 *
 * Threading: a context is bound to one CUDA device and one stream.  Calls on
 * one context must be externally serialised; separate contexts (one per GPU)
 * may be used from separate threads.
 *
 * Memory: every handle owns the device memory it allocates and frees it in
 * its *_destroy call.  Input arrays are copied during the create call.  Output
 * buffers are caller-provided; FF_MEM_DEVICE in a flags word says the pointer
 * is device memory of the context's device, otherwise it is host memory.
 */
#ifndef FIREFLY_B200_H
#define FIREFLY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FF_ABI_VERSION 1

#if defined(__GNUC__)
#define FF_API __attribute__((visibility("default")))
#else
#define FF_API
#endif

/* Status codes.  The reference terminates the process on any CUDA error
 * (CudaHelpers.cpp:3-11 checkCudaErrors -> exit(99); massert.cpp:3-12 ->
 * abort()); every call here returns one of these instead. */
typedef enum ff_status {
    FF_OK = 0,
    FF_ERR_INVALID_ARG = 1,
    FF_ERR_OOM = 2,
    FF_ERR_CUDA = 3,
    FF_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    FF_ERR_UNSUPPORTED = 5,
    FF_ERR_INTERNAL = 6
} ff_status;

typedef struct ff_context ff_context;
typedef struct ff_scene ff_scene;
typedef struct ff_film ff_film;

/* Pointer-location flags for buffers passed across the ABI. */
#define FF_MEM_HOST   0u
#define FF_MEM_DEVICE 1u

/* ---------------------------------------------------------------- context */

typedef struct ff_device_opts {
    int32_t device;       /* CUDA ordinal */
    void* stream;         /* cudaStream_t to run on; NULL = a stream owned by the context */
    uint32_t flags;       /* reserved, 0 */
} ff_device_opts;

/* Replaces PathTracer::init_interop's stream/event creation
 * (PathTracer.cpp:81-96) without the GL interop. */
FF_API ff_status ff_context_create(const ff_device_opts* opts, ff_context** out);
FF_API ff_status ff_context_destroy(ff_context* ctx);
/* Message of the last failed call on this context (never NULL). */
FF_API const char* ff_last_error_message(const ff_context* ctx);
/* Synchronise the context's stream. */
FF_API ff_status ff_context_sync(ff_context* ctx);
/* The stream the context launches on (a cudaStream_t). */
FF_API void* ff_context_stream(const ff_context* ctx);

/* ------------------------------------------------------------------ scene */

/* Material kinds.  FF_MAT_MIX is the reference's only wired material: the
 * 50/50 diffuse + GGX mixture of BRDF_L/BRDF_f/BRDF_pdf (dMaterial.cu:363-469).
 * FF_MAT_DIFFUSE and FF_MAT_CONDUCTOR are its single-lobe stages
 * (wf_mat_diffuse / wf_mat_cook, kernel.cu:546-614).  FF_MAT_DIELECTRIC and
 * FF_MAT_COAT have no counterpart in the reference (it defines refract() at
 * dMaterial.cu:97-113 but never uses it). */
typedef enum ff_material_kind {
    FF_MAT_MIX = 0,
    FF_MAT_DIFFUSE = 1,
    FF_MAT_CONDUCTOR = 2,
    FF_MAT_DIELECTRIC = 3,
    FF_MAT_COAT = 4
} ff_material_kind;

/* Flattened dMaterial (dMaterial.cuh:9-31): glTF metallic-roughness factors.
 * Textures are referenced by index into ff_scene_desc.textures, -1 = none,
 * and read as the reference's get_albedo / get_roughness / get_metallic /
 * get_normal read them (dMaterial.cu:10-88): the roughness from
 * metallic_roughness_tex channel 1 if set, else roughness_tex channel 0 (both
 * at least 0.01), else the factor; the metallic from metallic_roughness_tex
 * channel 2, else metallic_tex channel 0, else the factor; the shading normal
 * from normal_tex through the interpolated tangent frame (TBN * (2 t - 1)). */
typedef struct ff_material {
    float base_color[3];      /* baseColorFactor */
    float emissive[3];        /* emissiveColorFactor */
    float fresnel[3];         /* f0 of the dielectric part, default 0.04 */
    float roughness;          /* roughnessFactor */
    float metallic;           /* metallicFactor */
    float radiance;           /* emission scale, emissive_L = radiance * emissive */
    float ior;                /* FF_MAT_DIELECTRIC / FF_MAT_COAT only */
    int32_t kind;             /* ff_material_kind */
    int32_t base_color_tex;   /* baseColorTexture, -1 = none */
    int32_t roughness_tex;    /* roughnessTexture, -1 = none */
    int32_t metallic_tex;     /* metallicTexture, -1 = none */
    int32_t metallic_roughness_tex; /* metallicRoughnessTexture (glTF packing), -1 = none */
    int32_t normal_tex;       /* normalTexture (tangent space), -1 = none */
} ff_material;

/* RGB float texture, row-major, texel (x, y) at data[3*(y*width + x)]. */
typedef struct ff_texture_desc {
    const float* rgb;
    uint32_t width, height;
} ff_texture_desc;

/* Rectangular area light, the reference's _Rectangle (Rectangle.cuh:24-123)
 * wrapped by dAreaLight (dAreaLight.cu:18-68): p0 + s*a + t*b, s,t in [0,1]. */
typedef struct ff_area_light {
    float p0[3], a[3], b[3], normal[3];
    float emissive[3];        /* emissiveColorFactor of the light's material */
    float radiance;           /* radiance of the light's material */
} ff_area_light;

/* Directional light, the reference's dDirectionalLight (dDirectionalLight.cu:
 * 5-57): a delta light from `direction` (pointing from the scene toward the
 * light; normalised on upload), radiance * emissive, pdf 1, visibility by an
 * any-hit ray of unbounded length.  Added by add_directional_lights
 * (kernel.cu:725-731). */
typedef struct ff_directional_light {
    float direction[3];
    float emissive[3];
    float radiance;
    float pad;
} ff_directional_light;

/* dCamera (dCamera.cuh:9-22) with the inverse view-projection given directly
 * (the reference computes glm::inverse(P*V) on the host, dScene.cpp:381-391).
 * inv_view_proj is the reference's Matrix4x4 m[4][4] flattened row-major,
 * used as m * float4 (dMatrix.cuh:61-69). */
typedef struct ff_camera {
    float inv_view_proj[16];
    float lens_radius;        /* thin lens, 0 = pinhole */
    float focal_distance;     /* dCamera::f */
    float exposure;           /* dCamera::exposure_time */
    float pixel_jitter;       /* origin jitter scale, reference 0.005 (dCamera.cu:22) */
} ff_camera;

typedef struct ff_scene_desc {
    const float* positions;       /* float3 per vertex */
    uint32_t num_vertices;
    const uint32_t* indices;      /* uint3 per triangle */
    uint32_t num_triangles;
    const float* normals;         /* float3 per vertex, NULL = face normals */
    const float* texcoords;       /* float2 per vertex, NULL = zeros */
    const uint32_t* material_ids; /* per triangle, NULL = all 0 */
    const ff_material* materials;
    uint32_t num_materials;
    const ff_texture_desc* textures;
    uint32_t num_textures;
    /* Environment light (dEnvironmentLight): an equirectangular RGB32F map
     * (env_rgb != NULL) or a constant colour. */
    const float* env_rgb;
    uint32_t env_width, env_height;
    float env_color[3];
    const ff_area_light* area_lights;
    uint32_t num_area_lights;
    ff_camera camera;
    uint32_t flags;               /* reserved, 0 */
    const ff_directional_light* directional_lights;
    uint32_t num_directional_lights;
    /* Per-vertex tangent frame for normal textures (dVertex.cuh:4-10), float3
     * each; NULL = derived per triangle from positions and texcoords (the
     * reference takes assimp's aiProcess_CalcTangentSpace frame). */
    const float* tangents;
    const float* bitangents;
} ff_scene_desc;

typedef struct ff_scene_stats {
    uint32_t num_triangles;
    uint32_t num_nodes;           /* 8-wide BVH nodes */
    uint32_t num_leaf_refs;       /* triangle references stored in leaves */
    uint32_t bvh_depth;
    uint64_t device_bytes;        /* device memory held by the scene */
    float build_ms;               /* device BVH build time */
    float scene_lo[3], scene_hi[3];
} ff_scene_stats;

/* Replaces dScene::dScene(Scene*) and dScene::load_scene (dScene.cpp:19-23,
 * 60-80): materials, mesh flattening (process_mesh, kernel.cu:714-723),
 * camera, lights (add_environment_light kernel.cu:742-771, add_area_lights
 * kernel.cu:733-739) and the BVH (BVHAccel, dScene.cpp:364-379, plus
 * reorder_primitives kernel.cu:701-712).  The BVH is built on the device. */
FF_API ff_status ff_scene_create(ff_context* ctx, const ff_scene_desc* desc, ff_scene** out);
FF_API ff_status ff_scene_destroy(ff_scene* scene);
/* Replaces dScene::update / update_camera (dScene.cpp:55-58, 381-391). */
FF_API ff_status ff_scene_update_camera(ff_scene* scene, const ff_camera* camera);
FF_API ff_status ff_scene_get_stats(const ff_scene* scene, ff_scene_stats* out);

/* -------------------------------------------------------------- ray query */

/* A ray as the trace entry point consumes it (32 bytes).  The reference's
 * dRay (dRay.cuh:5-11) has no interval; tmin = 0, tmax = +inf reproduce it. */
typedef struct ff_ray {
    float ox, oy, oz, tmin;
    float dx, dy, dz, tmax;
} ff_ray;

/* Closest-hit result (16 bytes).  prim is the caller's ORIGINAL triangle
 * index (the reference reports the post-reorder index, dTriangle.cu:172;
 * orderedPrims maps it back, BVH.cpp:95-96), -1 on a miss, and -2 - index
 * for a back face of an FF_TRACE_TWO_SIDED query.  u weights the second
 * vertex and v the third, as in dTriangle::hit (dTriangle.cu:94-97). */
typedef struct ff_hit {
    float t, u, v;
    int32_t prim;
} ff_hit;

#define FF_TRACE_CLOSEST 0u   /* intersect(), dTriangle.cu:140-213 */
#define FF_TRACE_ANY     2u   /* intersect_shadows(), dTriangle.cu:215-259 */
/* Closest hits that also take back faces (no counterpart in the reference,
 * which culls them, dTriangle.cu:5,41): a back face passes the mirror image
 * of the culling test (determinant <= -1e-6, the same FP32 edge tests and FP64
 * epilogue on the negated determinant and numerators) and is reported as
 * prim = -2 - index; front faces give exactly the culling test's answers.
 * The path tracer traces rays inside refracting objects this way. */
#define FF_TRACE_TWO_SIDED 4u
/* Location of rays/hits: FF_MEM_DEVICE (bit 0) or host. */

/* Replaces wf_extend / wf_shadow (kernel.cu:488-543): trace n rays against
 * the scene.  Closest-hit follows dTriangle::intersect (culling Moller-Trumbore,
 * FP64 reciprocal of det) and returns the hit with the smallest t, ties to the
 * lowest original triangle index, counting hits with tmin <= t < min(tmax,1e32).
 * Any-hit follows dTriangle::shadow_hit (two-sided) and sets prim to the index
 * of some occluder with tmin <= t < tmax, or -1.  flags = FF_TRACE_* |
 * FF_MEM_DEVICE when rays and hits are device pointers.  With host pointers
 * the call copies in and out and returns after the hits are on the host. */
FF_API ff_status ff_trace(ff_context* ctx, const ff_scene* scene, const ff_ray* rays,
                   uint64_t n, ff_hit* hits, uint32_t flags);

/* Host-pointer ray query that allocates no device memory.  No counterpart in
 * the reference.  For callers that cannot allocate device memory: an
 * application whose device memory is owned by its own pool allocator under a
 * fixed budget, or an interactive loop that cannot take the implicit device
 * synchronisation of cudaMalloc / cudaFree (ff_trace's host path grows its
 * staging buffers with cudaMalloc).  Same query and results as ff_trace with
 * host pointers (flags: FF_TRACE_CLOSEST or FF_TRACE_ANY, FF_MEM_DEVICE is
 * rejected), for at most FF_NOALLOC_MAX_RAYS rays per call; larger n returns
 * FF_ERR_INVALID_ARG.  Its scratch is one fixed array of about 3 MiB in the
 * library's device image, held by every GPU that loads the library until the
 * process exits.  The first call on a device looks up that array's device
 * address and keeps it for the life of the process; make that first call
 * before any stream capture.  cudaDeviceReset invalidates that address
 * together with every context and scene of this library on the device, so
 * this entry point must not be called on a device after a reset.  All calls
 * on a device share the array: calls whose GPU work overlaps race and must
 * be serialised by the caller. */
#define FF_NOALLOC_MAX_RAYS 65536u
FF_API ff_status ff_trace_host_noalloc(ff_context* ctx, const ff_scene* scene, const ff_ray* rays,
                                       uint64_t n, ff_hit* hits, uint32_t flags);

/* Traversal work of n rays, for measurement; no counterpart in the
 * reference.  Runs the same traversal as ff_trace (same rays and flags,
 * FF_MEM_DEVICE when rays is a device pointer) without writing hits, and
 * returns out[0] = 8-wide node records fetched, out[1] = triangles tested,
 * out[2] = bytes per node record, out[3] = bytes per triangle record, so
 * that (out[0]*out[2] + out[1]*out[3]) / n is the traversal's fetched bytes
 * per ray.  Synchronous. */
FF_API ff_status ff_trace_count(ff_context* ctx, const ff_scene* scene, const ff_ray* rays,
                                uint64_t n, uint32_t flags, uint64_t* out);

/* ------------------------------------------------------------------- film */

/* Headless film replacing the GL surface of Interop (Interop.cpp:78-86) and
 * the accumulatebuffer / n_samples pair (PathTracer.cpp:22-23). */
FF_API ff_status ff_film_create(ff_context* ctx, uint32_t width, uint32_t height, ff_film** out);
FF_API ff_status ff_film_destroy(ff_film* film);
/* Replaces PathTracer::clear_buffer (PathTracer.cpp:150-170). */
FF_API ff_status ff_film_clear(ff_film* film);
/* Accumulated radiance (RGBA float, A = 0) and per-pixel sample counts.
 * Either pointer may be NULL.  flags: FF_MEM_DEVICE or host. */
FF_API ff_status ff_film_read(ff_film* film, float* rgba, uint32_t* n_samples, uint32_t flags);
/* Display image the way wf_logic writes its surface (kernel.cu:447-454):
 * accum/n * exposure, x/(1+x), then 8-bit.  rgba8 is width*height*4 bytes. */
FF_API ff_status ff_film_tonemap(ff_film* film, float exposure, uint8_t* rgba8, uint32_t flags);

/* ----------------------------------------------------------------- render */

#define FF_LIGHT_ALL (-2)      /* ff_render_settings.light: uniform light selection per vertex */
#define FF_RENDER_PROFILE 1u  /* ff_render_settings.flags: time every stage with CUDA events */

#define FF_MODE_PARITY    0u  /* reproduce the reference's behaviours (RR, MIS gating, offsets, env pdf) */
#define FF_MODE_CORRECTED 1u  /* unbiased RR, offset extension rays, fixed MIS gating */

typedef struct ff_render_settings {
    uint32_t spp;               /* samples per pixel added by this call */
    uint32_t max_depth;         /* MAX_PATH_LENGTH, reference 3 (PathTracer.h:21) */
    uint32_t rr_depth;          /* RR when path length > rr_depth, reference 3 (kernel.cu:372) */
    uint32_t seed;
    uint32_t mode;              /* FF_MODE_* */
    int32_t light;              /* -1 = environment, 0..A-1 = area light k, A..A+D-1 = directional light k-A,
                                   FF_LIGHT_ALL = one light per vertex chosen uniformly among all of them
                                   (corrected mode); the reference wires 1 = env (kernel.cu:397) */
    uint32_t max_paths;         /* path pool size, 0 = automatic */
    uint32_t sample_offset;     /* index of the first sample (progressive rendering) */
    uint32_t flags;             /* FF_RENDER_* */
    float shadow_offset;        /* SHADOW_OFFSET, reference 0.001 (kernel.cu:20) */
} ff_render_settings;

typedef struct ff_render_stats {
    uint64_t extension_rays;    /* closest-hit queries traced */
    uint64_t shadow_rays;       /* any-hit queries traced */
    uint64_t samples;           /* completed paths */
    uint32_t frames;            /* wavefront iterations */
    float ms_total;
    /* per-stage device time, filled with FF_RENDER_PROFILE */
    float ms_trace_extension, ms_trace_shadow, ms_logic, ms_shade;
    uint32_t kernel_launches;   /* kernels this call launched */
    /* ff_render_cached: device time of its stages (FF_RENDER_PROFILE) and the
     * cache queries answered and training records produced */
    float ms_cache_paths, ms_cache_train, ms_cache_query;
    uint64_t cache_queries, cache_records;
    /* ff_render_adjoint: texels touched by gradient atomics after the warp
     * pre-reduction (3 float atomics = 12 B each) */
    uint64_t grad_atomics;
    /* ff_render_adjoint: roughness texels touched (1 float atomic = 4 B each) */
    uint64_t grad_atomics_roughness;
    /* ff_render with FF_RENDER_PROFILE: the traversal work of the traced
     * rays, counted by a second pass of the same traversal over each frame's
     * queues (8-wide node records fetched, triangles tested; a node record is
     * 80 B, a triangle record 48 B) */
    uint64_t ext_nodes, ext_tris, shadow_nodes, shadow_tris;
} ff_render_stats;

/* Replaces PathTracer::draw + wavefront_pathtrace (PathTracer.cpp:59-79,
 * kernel.cu:658-676): run the wavefront until every pixel of the film has
 * received settings->spp more samples.  stats may be NULL. */
FF_API ff_status ff_render(ff_context* ctx, ff_scene* scene, const ff_render_settings* settings,
                    ff_film* film, ff_render_stats* stats);

/* -------------------------------------------------------------- adjoint */

#define FF_ADJOINT_STORE_ALL 4u   /* ff_adjoint_desc.flags: store-all-vertices reference variant */
#define FF_ADJOINT_MEGAKERNEL 16u /* ff_adjoint_desc.flags: one-thread-per-sample replay (cross-check) instead of
                                     the wavefront replay */
#define FF_ENV_KEEP_TABLES   8u   /* ff_scene_set_environment: keep the importance tables */

/* Gradient request of ff_render_adjoint.  d_image is dL/dI for the mean
 * radiance image I (width*height*3 floats).  Gradients are ADDED to
 * grad_texture (texels*3 floats of texture `texture`), grad_env
 * (env texels*3 floats) and grad_roughness (texels*3 floats of texture
 * `roughness_texture`: channel x where a material reads it as its
 * roughness_tex, channel y where it is the material's packed
 * metallic_roughness_tex; channel z, metallic, receives none).  flags: FF_MEM_DEVICE when every pointer is
 * device memory, FF_ADJOINT_STORE_ALL for the store-all reference variant. */
typedef struct ff_adjoint_desc {
    uint32_t width, height;
    const float* d_image;
    int32_t texture;          /* albedo texture receiving gradients, -1 = none */
    float* grad_texture;
    float* grad_env;          /* NULL = no environment gradient */
    uint32_t flags;
    int32_t roughness_texture; /* read only when grad_roughness != NULL */
    float* grad_roughness;    /* NULL = no roughness gradient */
} ff_adjoint_desc;

/* Path-replay adjoint of ff_render (no counterpart in the reference, which
 * renders only): the same paths as ff_render in FF_MODE_CORRECTED for the same
 * settings (seed, spp, sample_offset, depths, light), replayed from their
 * seeds; gradients of the albedo texture of FF_MAT_DIFFUSE surfaces, of the
 * roughness texture of GGX surfaces (FF_MAT_MIX, CONDUCTOR, DIELECTRIC, COAT)
 * and of the environment map (camera misses and NEE), with detached sampling
 * (directions, pdfs, MIS weights and the roulette are not differentiated).
 * settings->mode must be FF_MODE_CORRECTED.  stats: rays traced, samples,
 * device time. */
FF_API ff_status ff_render_adjoint(ff_context* ctx, ff_scene* scene, const ff_render_settings* settings,
                                   const ff_adjoint_desc* desc, ff_render_stats* stats);

/* Replace the texels of texture `index` (same size; width*height*3 floats).
 * flags: FF_MEM_DEVICE for a device pointer.  No counterpart in the reference,
 * whose textures are immutable CUDA texture objects (dTexture.cu:21-111). */
FF_API ff_status ff_scene_set_texture(ff_scene* scene, uint32_t index, const float* rgb, uint32_t flags);

/* Replace the environment map's texels (same size) and rebuild its
 * importance tables, unless flags has FF_ENV_KEEP_TABLES.  flags may also hold
 * FF_MEM_DEVICE.  No counterpart in the reference (add_environment_light,
 * kernel.cu:742-771, runs once at scene load). */
FF_API ff_status ff_scene_set_environment(ff_scene* scene, const float* rgb, uint32_t flags);

/* Adam hyper-parameters and step number (from 1); the parameter is clamped
 * to [lo, hi] after the update. */
typedef struct ff_adam_params {
    float lr, beta1, beta2, eps, lo, hi;
    uint32_t step;
} ff_adam_params;

/* One Adam update of n device floats on the context's stream (asynchronous),
 * for inverse rendering with ff_render_adjoint.  No counterpart in the
 * reference.  param, grad, m, v are device pointers. */
FF_API ff_status ff_optimizer_adam_step(ff_context* ctx, float* param, const float* grad, float* m, float* v,
                                        uint64_t n, const ff_adam_params* hp);

/* Environment-map importance tables (kernel.cu:65-149): the marginal CDF
 * (height doubles), the conditional CDFs (height*width doubles, row-major) and
 * the pdf texture (height*width floats, already scaled by w*h/(2*pi^2)), as
 * the device scans produced them.  Any pointer may be NULL.  Host memory. */
FF_API ff_status ff_scene_read_env_tables(const ff_scene* scene, double* marginal, double* conditional,
                                   float* pdf, double* pdf_denom);

/* No counterpart in the reference: the scene's 8-wide BVH as ff_trace walks
 * it, copied to host memory for inspection and tests.  nodes receives
 * *num_nodes records of 80 bytes: origin (3 floats), three biased exponents
 * and the internal-child mask (4 bytes), the first internal child and the
 * first triangle (2 uint32), per slot a meta byte (0 empty; internal 0x20 |
 * 24 + slot; leaf: unary triangle count << 5 | offset from the first
 * triangle), then the quantised planes lo x, y, z and hi x, y, z (8 bytes
 * each).  tris receives *num_tris records of 48 bytes in leaf order: v0 with
 * the original index as the fourth word's bits, e1 = v1 - v0, e2 = v2 - v0
 * (each padded to 4 floats).  With nodes or tris NULL only the counts are
 * written; a capacity (bytes) below the size returns FF_ERR_INVALID_ARG. */
FF_API ff_status ff_scene_read_bvh(const ff_scene* scene, void* nodes, uint64_t nodes_capacity, void* tris,
                                   uint64_t tris_capacity, uint32_t* num_nodes, uint32_t* num_tris);

/* ------------------------------------------------------------------------
 * Learned radiance cache (no counterpart in the reference).  A multiresolution
 * hash grid (FF_CACHE_LEVELS levels x 2 features, 2^log2_table_size entries per
 * level, resolutions from base_resolution to max_resolution cells across the
 * scene box) and an MLP of 4 hidden ReLU layers of 64 units with 3 outputs,
 * bf16 weights and FP32 accumulation on the tensor cores.  Inputs: the hash
 * features of the position, degree-4 spherical harmonics of the outgoing
 * direction, the normal, the roughness and a constant 1.  Trained with Adam on
 * the relative L2 loss sum_c (y_c - t_c)^2 / (y_c^2 + 0.01), mean over records.
 * ------------------------------------------------------------------------ */
typedef struct ff_cache ff_cache;

#define FF_CACHE_LEVELS 16
#define FF_CACHE_MLP_PARAMS (5 * 64 * 64)  /* W0..W3 [64][64], W4 [64][64] with rows 3..63 zero; W[out][in] */

typedef struct ff_cache_params {
    uint32_t log2_table_size;   /* entries per level = 2^log2_table_size (19) */
    uint32_t base_resolution;   /* cells across the box at level 0 (16) */
    uint32_t max_resolution;    /* cells across the box at the last level (2048) */
    uint32_t seed;              /* parameter initialisation */
    float lr, beta1, beta2, eps;    /* Adam */
    float rough_threshold;      /* ff_render_cached: roughness at or above which a vertex is rough */
    uint32_t train_paths;       /* ff_render_cached: training paths per frame (65536) */
    uint32_t train_batch;       /* ff_render_cached: records per optimiser step (16384) */
    uint32_t flags;             /* reserved, 0 */
} ff_cache_params;

/* One cache record: a path vertex and a value (training: the target radiance
 * leaving the vertex toward wo; render queries: the path throughput). */
typedef struct ff_cache_record {
    float pos[3];               /* world space */
    float roughness;
    float wo[3];                /* unit direction toward the previous vertex */
    float value_r;
    float normal[3];
    float value_g;
    uint32_t pixel;             /* render queries: film pixel */
    float value_b;
    float pad[2];
} ff_cache_record;              /* 64 bytes */

#define FF_CACHE_GRADIENTS_ONLY 16u  /* ff_cache_train: accumulate gradients, take no optimiser step */

/* The cache's box is the scene's bounding box. */
FF_API ff_status ff_cache_create(ff_context* ctx, const ff_scene* scene, const ff_cache_params* params,
                                 ff_cache** out);
FF_API ff_status ff_cache_destroy(ff_cache* cache);
/* Re-initialise every parameter and the optimiser state. */
FF_API ff_status ff_cache_reset(ff_cache* cache);
/* rgb[3*i..] = the MLP's output for record i.  flags: FF_MEM_DEVICE when both
 * pointers are device memory. */
FF_API ff_status ff_cache_query(ff_cache* cache, const ff_cache_record* records, uint32_t n, float* rgb,
                                uint32_t flags);
/* One optimiser step on the n records (their value = target radiance), or
 * only the gradients with FF_CACHE_GRADIENTS_ONLY.  loss (host, may be NULL)
 * receives the batch's mean relative L2 loss. */
FF_API ff_status ff_cache_train(ff_cache* cache, const ff_cache_record* records, uint32_t n, uint32_t flags,
                                float* loss);
/* FP32 parameters and gradient accumulators (host memory, any may be NULL):
 * mlp and grad_mlp FF_CACHE_MLP_PARAMS floats, grid and grad_grid
 * FF_CACHE_LEVELS * 2^log2_table_size * 2 floats. */
FF_API ff_status ff_cache_read_params(ff_cache* cache, float* mlp, float* grid, float* grad_mlp, float* grad_grid);
FF_API ff_status ff_cache_write_params(ff_cache* cache, const float* mlp, const float* grid);
/* Render settings->spp frames of one path per pixel each into the film:
 * paths run as in ff_render (corrected mode) up to the first rough vertex
 * after the camera hit, where they end with throughput x the cache's radiance;
 * settings->max_depth bounds specular chains.  Every frame also traces
 * params.train_paths full-length training paths from random pixels, whose
 * radiance from their first rough vertex on trains the cache (one or more
 * optimiser steps of train_batch records) after the frame's queries. */
FF_API ff_status ff_render_cached(ff_context* ctx, ff_scene* scene, ff_cache* cache,
                                  const ff_render_settings* settings, ff_film* film, ff_render_stats* stats);

/* ------------------------------------------------------------------------
 * Test hooks (no counterpart in the reference, whose checkCudaErrors exits
 * the process, CudaHelpers.cpp:3-11): they drive the error paths that
 * replace exit(99) without faulting or hanging a GPU.
 * ------------------------------------------------------------------------ */
#define FF_DEBUG_WAIT_DEFAULT 0xffffffffu

/* Device allocations this library made since it was loaded (total) and the
 * ones it still holds (live), over all contexts.  Either pointer may be NULL. */
FF_API ff_status ff_debug_alloc_stats(uint64_t* total, int64_t* live);
/* From now on the next n device allocations of this library succeed and
 * every later one fails with FF_ERR_OOM, without calling cudaMalloc; n < 0
 * turns the refusal off.  Process-wide. */
FF_API ff_status ff_debug_fail_alloc_after(int64_t n);
/* Bound of the radiance cache's tensor-core waits, in polls of the
 * mbarrier (0: every wait gives up at once; FF_DEBUG_WAIT_DEFAULT: the
 * built-in bound).  A wait that gives up makes the call return
 * FF_ERR_TIMEOUT; the kernel first waits, with the built-in bound, for the
 * tensor-core work it issued, then frees its tensor memory. */
FF_API ff_status ff_debug_cache_wait_limit(ff_cache* cache, uint32_t polls);
/* The texel the environment light's importance sampling picks for each of
 * n draw pairs (ex, ey) (host array of 2n floats): the two CDF searches of
 * get_direction (CUDA-RayTracer/dEnvironmentLight.cu:41-58) as the path
 * kernels run them, guide tables included, on the device.  xy (host, 2n
 * int32) receives the column x and row y of each pick.  For tests of the
 * searches against the tables of ff_scene_read_env_tables. */
FF_API ff_status ff_debug_env_pick(const ff_scene* scene, const float* exy, uint64_t n, int32_t* xy);

#ifdef __cplusplus
}
#endif

#endif /* FIREFLY_B200_H */
