// ff_internal.h — host-side objects behind the opaque handles of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "ff_cache.cuh"
#include "ff_common.cuh"
#include "firefly_b200.h"

// Deepest 8-wide BVH the traversal stack can serve (checked at scene build).
constexpr int kMaxStackDepth = 64;

// Raised inside the implementation and turned into an ff_status at the ABI.
struct FFError {
    ff_status status;
    std::string msg;
};

#define FF_CUDA_CHECK(expr)                                                              \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess) {                                                         \
            throw FFError{_e == cudaErrorMemoryAllocation ? FF_ERR_OOM : FF_ERR_CUDA,    \
                          std::string(#expr) + ": " + cudaGetErrorString(_e)};           \
        }                                                                                \
    } while (0)

#define FF_REQUIRE(cond, msg)                                  \
    do {                                                       \
        if (!(cond)) throw FFError{FF_ERR_INVALID_ARG, (msg)}; \
    } while (0)

// Device allocations made through DevBuf, process-wide (ff_debug_alloc_stats),
// and the test hook that refuses them (ff_debug_fail_alloc_after): while
// fail_after >= 0, that many more allocations succeed and every later one
// fails with FF_ERR_OOM without reaching cudaMalloc.
struct FFAllocStats {
    std::atomic<uint64_t> total{0};
    std::atomic<int64_t> live{0};
    std::atomic<int64_t> fail_after{-1};
};
extern FFAllocStats g_ff_alloc;

inline bool ff_alloc_refused()
{
    int64_t left = g_ff_alloc.fail_after.load();
    while (left >= 0) {
        if (left == 0) return true;
        if (g_ff_alloc.fail_after.compare_exchange_weak(left, left - 1)) return false;
    }
    return false;
}

// Owning device allocation.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (ptr) {
            cudaFree(ptr);
            g_ff_alloc.live.fetch_sub(1);
        }
        ptr = nullptr;
        bytes = 0;
    }
    void alloc(size_t n)
    {
        if (n <= bytes && ptr) return;
        release();
        if (n == 0) return;
        if (ff_alloc_refused()) throw FFError{FF_ERR_OOM, "device allocation refused (ff_debug_fail_alloc_after)"};
        FF_CUDA_CHECK(cudaMalloc(&ptr, n));
        g_ff_alloc.total.fetch_add(1);
        g_ff_alloc.live.fetch_add(1);
        bytes = n;
    }
    template <class T>
    T* as() const { return reinterpret_cast<T*>(ptr); }
};

struct FFWavefrontWS;
void ff_wavefront_ws_free(FFWavefrontWS* ws);

struct ff_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int num_sms = 148;
    std::string last_error;
    DevBuf counters;      // small scratch of uint32 counters for persistent kernels
    DevBuf io_rays, io_hits;  // staging for host-pointer ff_trace calls
    // host-pointer ff_trace: rays copied in on io_in, hits copied out on
    // io_out, each chunk's trace on `stream` between them (created on first use)
    cudaStream_t io_in = nullptr, io_out = nullptr;
    cudaEvent_t io_ev_start = nullptr, io_ev_in = nullptr, io_ev_traced = nullptr;
    DevBuf adj_io[5];         // ff_render_adjoint: staged image, texture / env / roughness gradients, counters
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    FFWavefrontWS* adj_ws = nullptr;   // path pool of ff_render_adjoint, kept between calls
    // resident blocks per SM of each queue-driven k_trace variant on this
    // context's device (0 = not yet queried), indexed by any-hit | tagged << 1 | two-sided << 2
    int trace_bps[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// Per-original-triangle shading attributes, read once per hit by a gather
// over the triangle index: the three vertex normals, the material index and
// the three texture coordinates in four 16-byte loads, padded to an 80-byte
// stride.  (Packed to 64 bytes, the same fields made k_logic 23% slower on
// the 1.3M-triangle scene, 96.4 against 78.4 ms per 64-spp step, measured
// on one box back to back.)
struct __align__(16) FFShadeTri {
    float n0x, n0y, n0z, n1x;
    float n1y, n1z, n2x, n2y;
    float n2z;
    uint32_t material;
    float u0, v0;
    float u1, v1, u2, v2;
    float pad[4];
};
static_assert(sizeof(FFShadeTri) == 80, "80-byte stride");

struct FFShadeRec {
    float3 n0, n1, n2;   // vertex normals
    float2 uv0, uv1, uv2;
    uint32_t material;
};
#ifdef __CUDACC__
__device__ __forceinline__ FFShadeRec ff_load_shade(const FFShadeTri* __restrict__ tris, uint32_t i)
{
    const float4* q = reinterpret_cast<const float4*>(tris + i);
    const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
    FFShadeRec r;
    r.n0 = make_float3(a.x, a.y, a.z);
    r.n1 = make_float3(a.w, b.x, b.y);
    r.n2 = make_float3(b.z, b.w, c.x);
    r.material = __float_as_uint(c.y);
    r.uv0 = make_float2(c.z, c.w);
    r.uv1 = make_float2(d.x, d.y);
    r.uv2 = make_float2(d.z, d.w);
    return r;
}
#endif

struct FFEnvLight {
    int width = 0, height = 0;
    float3 color = {1.f, 1.f, 1.f};
    DevBuf rgb;           // float3 texels (width*height)
    DevBuf marginal;      // double[height]
    DevBuf conditional;   // double[height*width]
    DevBuf pdf;           // float[height*width]
    DevBuf denom;         // double
    DevBuf texel4;        // float4[height*width]: rgb and pdf packed for the path kernels
    DevBuf guide;         // uint32: the marginal's search guide, then one per conditional row
};

struct ff_scene {
    ff_context* ctx = nullptr;
    uint32_t num_tris = 0;
    uint32_t num_nodes = 0;
    uint32_t depth = 0;
    float build_ms = 0.f;
    float3 lo{0, 0, 0}, hi{0, 0, 0};
    DevBuf nodes;         // FFNode8[num_nodes]
    DevBuf tris;          // FFTri[num_tris] in leaf order
    DevBuf shade;         // FFShadeTri[num_tris] by original index
    DevBuf tangent;       // FFTangentTri[num_tris] when a material has a normal texture, else empty
    DevBuf materials;     // ff_material[num_materials]
    uint32_t num_materials = 0;
    std::vector<DevBuf*> textures;
    DevBuf tex_table;     // device table of texture descriptors
    DevBuf area_lights;   // ff_area_light[]
    uint32_t num_area_lights = 0;
    DevBuf dir_lights;    // ff_directional_light[], directions normalised
    uint32_t num_dir_lights = 0;
    FFEnvLight env;
    ff_camera camera{};
    // some material refracts (FF_MAT_DIELECTRIC): paths can run inside
    // objects, and the path tracer traces closest hits two-sided there
    bool refracts = false;
    ~ff_scene()
    {
        for (auto* t : textures) delete t;
    }
    FFBvhView view() const
    {
        return FFBvhView{nodes.as<FFNode8>(), tris.as<FFTri>(), num_nodes, num_tris};
    }
    size_t device_bytes() const;
};

struct ff_film {
    ff_context* ctx = nullptr;
    uint32_t width = 0, height = 0;
    DevBuf accum;         // float4 per pixel: radiance sum (xyz)
    DevBuf comp;          // float4 per pixel: Kahan compensation
    DevBuf count;         // uint32 per pixel
    DevBuf staging;       // float4 per pixel: resolved image / tonemapped bytes on their way to the host
    FFWavefrontWS* ws = nullptr;  // path pool and queues of ff_render, kept between calls
    ~ff_film() { ff_wavefront_ws_free(ws); }
};

// ff_wavefront.cu.  With a cache hook, paths end at their first rough vertex
// after the camera hit with a query record (slot index as the pixel), and the
// cache's answers join the slot sums before the film update.
struct ff_cache;
struct FFCacheHook {
    ff_cache* cache;
    void* queries;            // ffc::Record[capacity]
    uint32_t* n_queries;      // device counter
    uint32_t capacity;
    float rough_threshold;
    cudaEvent_t ev_query0, ev_query1;   // recorded around the inference when not null
    cudaEvent_t wait_before_query;      // the stream waits for it before the inference when not null
};
void ff_wavefront_render(ff_context* ctx, ff_scene* scene, const ff_render_settings* st, ff_film* film,
                         ff_render_stats* stats, const FFCacheHook* hook = nullptr);

// ff_bvh.cu: device BVH build from host or device triangle data already on
// the device (positions float3[V], indices uint3[T]).
void ff_build_bvh(ff_context* ctx, ff_scene* s, const float3* d_pos, const uint3* d_idx,
                  uint32_t num_tris);

// ff_trace.cu
void ff_launch_trace(ff_context* ctx, const ff_scene* s, const ff_ray* d_rays, uint64_t n,
                     ff_hit* d_hits, bool any_hit, bool two_sided = false);
// ff_trace.cu: traversal work counts of n device rays (ff_trace_count):
// d_out[0] += node records fetched, d_out[1] += triangles tested.
void ff_launch_trace_count(ff_context* ctx, const ff_scene* s, const ff_ray* d_rays, uint64_t n, bool any_hit,
                           unsigned long long* d_out, unsigned int* err, bool two_sided = false);

// ff_trace.cu: traversal work counts of a device queue (the same traversal
// as ff_launch_trace_queue): d_out[0] += node records, d_out[1] += triangles.
void ff_launch_trace_count_queue(ff_context* ctx, const FFBvhView& bvh, const ff_ray* d_rays, const uint32_t* n_dev,
                                 uint64_t cap, bool any_hit, bool two_sided, unsigned long long* d_out,
                                 unsigned int* err, cudaStream_t stream);

// ff_trace.cu: the trace launch with caller-supplied counters (used by the
// no-allocation entry point).
void ff_launch_trace_scratch(ff_context* ctx, const ff_scene* s, const ff_ray* d_rays, uint64_t n,
                             ff_hit* d_hits, bool any_hit, unsigned long long* counter, unsigned int* err);

// ff_trace.cu: trace a device queue whose length is in device memory; with
// tags, closest hits go to d_hits[tag] and any-hit answers to occ[tag].
void ff_launch_trace_queue(ff_context* ctx, const FFBvhView& bvh, const ff_ray* d_rays, const uint32_t* n_dev,
                           uint64_t cap, ff_hit* d_hits, bool any_hit, unsigned long long* counter,
                           unsigned int* err, const uint32_t* tags = nullptr, uint8_t* occ = nullptr,
                           cudaStream_t stream = nullptr,   // null: the context's stream
                           bool two_sided = false,
                           int max_blocks_per_sm = 0);      // 0: as many as fit (the grid fills the GPU)          // honour the per-ray two-sided mark

// ff_wavefront.cu: the path-replay adjoint on the wavefront stages.  Every
// pointer is device memory; gradients are added to grad_* (null = not
// requested); touched[0..1] count the texels the atomics touched.
struct FFAdjointTarget {
    uint32_t width, height;
    const float* d_image;
    int32_t texture;
    float* grad_tex;
    float* grad_env;
    int32_t rough_texture;
    float* grad_rough;
    unsigned long long* touched;
};
void ff_wavefront_adjoint(ff_context* ctx, ff_scene* scene, const ff_render_settings* st, const FFAdjointTarget& t,
                          ff_render_stats* stats);

// ff_adjoint.cu
void ff_adjoint_render(ff_context* ctx, ff_scene* scene, const ff_render_settings* st, const ff_adjoint_desc* ad,
                       ff_render_stats* stats);
void ff_build_env_tables(ff_context* ctx, ff_scene* s);

// ff_scene.cu: device views of the scene's lights for the path kernels.
namespace ffp {
struct FFLightSet;
}
struct FFEnvView;
FFEnvView ff_env_view(const ff_scene* s);
void ff_check_light(const ff_scene* s, int32_t light, uint32_t mode);   // FF_REQUIRE on bad indices
ffp::FFLightSet ff_light_set(const ff_scene* s, int32_t light, uint32_t mode);

// ff_cache.cu: learned radiance cache.
struct ff_cache {
    ff_context* ctx = nullptr;
    ff_cache_params prm{};
    float3 lo{0, 0, 0}, hi{0, 0, 0};  // scene box
    ffc::Grid grid{};
    DevBuf table, table_h, grid_grad, grid_m, grid_v;   // float2 / half2 per grid entry
    DevBuf mlp, mlp_img, mlp_grad, mlp_m, mlp_v;        // FP32 weights, their bf16 images, Adam state
    DevBuf loss;          // float: sum of training losses since the last reset of the counter
    DevBuf err;           // uint32: tensor-core waits that gave up
    uint32_t wait_polls = FF_DEBUG_WAIT_DEFAULT;   // ff_debug_cache_wait_limit
    uint32_t step = 0;    // Adam steps taken
    // ff_render_cached workspace: training runs on `aux`, beside the pixel
    // paths on the context's stream
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_frame = nullptr, ev_trained = nullptr;
    DevBuf queries, train_recs, frame, counters;
    uint32_t ws_pixels = 0, ws_train = 0;
    DevBuf io_recs, io_out;   // staging for host-pointer calls
    ~ff_cache()
    {
        if (aux) {
            cudaStreamSynchronize(aux);
            cudaStreamDestroy(aux);
        }
        if (ev_frame) cudaEventDestroy(ev_frame);
        if (ev_trained) cudaEventDestroy(ev_trained);
    }
};
void ff_cache_setup_grid(ff_cache* c);
void ff_cache_init_params(ff_cache* c);
void ff_cache_refresh_copies(ff_cache* c);
uint32_t ff_cache_num_params();
void ff_cache_launch_infer(ff_cache* c, const void* recs, uint32_t n_max, const uint32_t* n_dev, float* out_rgb,
                           float4* frame);
void ff_cache_launch_train(ff_cache* c, const void* recs, uint32_t n, bool gradients_only);
void ff_cache_launch_train_slice(ff_cache* c, const void* recs, uint32_t offset, uint32_t n_max, const uint32_t* n_dev,
                                 cudaStream_t st);
void ff_cached_render(ff_context* ctx, ff_scene* scene, ff_cache* cache, const ff_render_settings* st, ff_film* film,
                      ff_render_stats* stats);
