// ff_api.cu — the extern "C" entry points declared in include/firefly_b200.h.
//
// Every entry point catches FFError and CUDA failures and returns an
// ff_status; nothing here exits or aborts the process (the reference calls
// exit(99) from checkCudaErrors, CUDA-RayTracer/CudaHelpers.cpp:3-11).
#include <algorithm>
#include <cstring>
#include <new>

#include "ff_internal.h"

namespace {

thread_local std::string g_create_error;

template <class F>
ff_status guarded(ff_context* ctx, F&& f)
{
    try {
        f();
        return FF_OK;
    } catch (const FFError& e) {
        if (ctx) ctx->last_error = e.msg;
        else g_create_error = e.msg;
        return e.status;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->last_error = "host allocation failed";
        return FF_ERR_OOM;
    } catch (...) {
        if (ctx) ctx->last_error = "unknown internal error";
        return FF_ERR_INTERNAL;
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) FF_CUDA_CHECK(cudaSetDevice(dev));
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

void upload(DevBuf& b, const void* host, size_t bytes, cudaStream_t st)
{
    b.alloc(bytes);
    if (bytes) FF_CUDA_CHECK(cudaMemcpyAsync(b.ptr, host, bytes, cudaMemcpyHostToDevice, st));
}

}  // namespace

size_t ff_scene::device_bytes() const
{
    size_t total = nodes.bytes + tris.bytes + shade.bytes + materials.bytes + tex_table.bytes + area_lights.bytes + dir_lights.bytes +
                   env.rgb.bytes + env.marginal.bytes + env.conditional.bytes + env.pdf.bytes + env.denom.bytes + env.texel4.bytes;
    for (auto* t : textures) total += t->bytes;
    return total;
}

// Defined in ff_envmap.cu and ff_scene.cu.
void ff_build_env_tables(ff_context* ctx, ff_scene* s);
void ff_env_pack(ff_context* ctx, ff_scene* s);
void ff_build_shading(ff_context* ctx, ff_scene* s, const ff_scene_desc* d, const float3* d_pos,
                      const uint3* d_idx);

extern "C" {

ff_status ff_context_create(const ff_device_opts* opts, ff_context** out)
{
    if (!out) return FF_ERR_INVALID_ARG;
    *out = nullptr;
    ff_context* ctx = new (std::nothrow) ff_context();
    if (!ctx) return FF_ERR_OOM;
    ff_status st = guarded(nullptr, [&] {
        int ndev = 0;
        FF_CUDA_CHECK(cudaGetDeviceCount(&ndev));
        int dev = opts ? opts->device : 0;
        FF_REQUIRE(dev >= 0 && dev < ndev, "device ordinal out of range");
        ctx->device = dev;
        DeviceGuard g(dev);
        FF_CUDA_CHECK(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, dev));
        if (opts && opts->stream) {
            ctx->stream = reinterpret_cast<cudaStream_t>(opts->stream);
            ctx->own_stream = false;
        } else {
            FF_CUDA_CHECK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
            ctx->own_stream = true;
        }
        ctx->counters.alloc(256);
        FF_CUDA_CHECK(cudaMemsetAsync(ctx->counters.ptr, 0, 256, ctx->stream));
        FF_CUDA_CHECK(cudaEventCreate(&ctx->ev0));
        FF_CUDA_CHECK(cudaEventCreate(&ctx->ev1));
    });
    if (st != FF_OK) {
        ff_context_destroy(ctx);   // the stream, events and buffers created before the failure
        return st;
    }
    *out = ctx;
    return FF_OK;
}

ff_status ff_context_destroy(ff_context* ctx)
{
    if (!ctx) return FF_ERR_INVALID_ARG;
    {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(ctx->device);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        ctx->counters.release();
        ctx->io_rays.release();
        ctx->io_hits.release();
        for (auto& b : ctx->adj_io) b.release();
        if (ctx->io_in) cudaStreamSynchronize(ctx->io_in);
        if (ctx->io_out) cudaStreamSynchronize(ctx->io_out);
        for (cudaEvent_t e : {ctx->io_ev_start, ctx->io_ev_in, ctx->io_ev_traced})
            if (e) cudaEventDestroy(e);
        if (ctx->io_in) cudaStreamDestroy(ctx->io_in);
        if (ctx->io_out) cudaStreamDestroy(ctx->io_out);
        if (ctx->ev0) cudaEventDestroy(ctx->ev0);
        if (ctx->ev1) cudaEventDestroy(ctx->ev1);
        ff_wavefront_ws_free(ctx->adj_ws);
        ctx->adj_ws = nullptr;
        if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
        if (prev >= 0) cudaSetDevice(prev);
    }
    delete ctx;
    return FF_OK;
}

const char* ff_last_error_message(const ff_context* ctx)
{
    if (!ctx) return g_create_error.c_str();
    return ctx->last_error.c_str();
}

ff_status ff_context_sync(ff_context* ctx)
{
    if (!ctx) return FF_ERR_INVALID_ARG;
    return guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        FF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

void* ff_context_stream(const ff_context* ctx) { return ctx ? reinterpret_cast<void*>(ctx->stream) : nullptr; }

ff_status ff_scene_create(ff_context* ctx, const ff_scene_desc* d, ff_scene** out)
{
    if (!ctx || !d || !out) return FF_ERR_INVALID_ARG;
    *out = nullptr;
    ff_scene* s = new (std::nothrow) ff_scene();
    if (!s) return FF_ERR_OOM;
    s->ctx = ctx;
    ff_status st = guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        FF_REQUIRE(d->num_triangles == 0 || (d->positions && d->indices), "positions and indices are required");
        FF_REQUIRE(d->num_triangles == 0 || d->num_vertices > 0, "num_vertices must be > 0");
        FF_REQUIRE(d->num_triangles < (1u << 30), "too many triangles");
        for (uint64_t i = 0; i < 3ull * d->num_triangles; ++i)
            FF_REQUIRE(d->indices[i] < d->num_vertices, "triangle index out of range");
        if (d->material_ids) {
            for (uint32_t i = 0; i < d->num_triangles; ++i)
                FF_REQUIRE(d->material_ids[i] < (d->num_materials ? d->num_materials : 1u),
                           "material id out of range");
        }
        FF_REQUIRE(d->num_materials < (1u << 24), "at most 2^24 - 1 materials");
        for (uint32_t m = 0; m < d->num_materials; ++m) {
            const ff_material& mt = d->materials[m];
            FF_REQUIRE(mt.kind >= FF_MAT_MIX && mt.kind <= FF_MAT_COAT, "unknown material kind");
            if (mt.kind == FF_MAT_DIELECTRIC) s->refracts = true;
            FF_REQUIRE(mt.base_color_tex < (int32_t)d->num_textures, "texture index out of range");
            FF_REQUIRE(mt.roughness_tex < (int32_t)d->num_textures, "texture index out of range");
        }
        FF_REQUIRE(!d->env_rgb || (d->env_width > 0 && d->env_height > 0), "environment map has zero size");
        FF_REQUIRE(d->num_area_lights == 0 || d->area_lights, "area_lights is NULL");
        FF_REQUIRE(d->num_directional_lights == 0 || d->directional_lights, "directional_lights is NULL");
        cudaStream_t stream = ctx->stream;
        DevBuf pos, idx;
        upload(pos, d->positions, sizeof(float) * 3ull * d->num_vertices, stream);
        upload(idx, d->indices, sizeof(uint32_t) * 3ull * d->num_triangles, stream);
        ff_build_bvh(ctx, s, pos.as<float3>(), idx.as<uint3>(), d->num_triangles);
        FF_REQUIRE(s->depth <= (uint32_t)kMaxStackDepth, "BVH deeper than the traversal stack");
        ff_build_shading(ctx, s, d, pos.as<float3>(), idx.as<uint3>());
        s->camera = d->camera;
        FF_CUDA_CHECK(cudaStreamSynchronize(stream));
    });
    if (st != FF_OK) {
        delete s;
        return st;
    }
    *out = s;
    return FF_OK;
}

ff_status ff_scene_destroy(ff_scene* s)
{
    if (!s) return FF_ERR_INVALID_ARG;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    delete s;
    if (prev >= 0) cudaSetDevice(prev);
    return FF_OK;
}

ff_status ff_scene_update_camera(ff_scene* s, const ff_camera* cam)
{
    if (!s || !cam) return FF_ERR_INVALID_ARG;
    s->camera = *cam;
    return FF_OK;
}

ff_status ff_scene_get_stats(const ff_scene* s, ff_scene_stats* out)
{
    if (!s || !out) return FF_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    out->num_triangles = s->num_tris;
    out->num_nodes = s->num_nodes;
    out->num_leaf_refs = s->num_tris;
    out->bvh_depth = s->depth;
    out->device_bytes = s->device_bytes();
    out->build_ms = s->build_ms;
    out->scene_lo[0] = s->lo.x;
    out->scene_lo[1] = s->lo.y;
    out->scene_lo[2] = s->lo.z;
    out->scene_hi[0] = s->hi.x;
    out->scene_hi[1] = s->hi.y;
    out->scene_hi[2] = s->hi.z;
    return FF_OK;
}

ff_status ff_scene_read_bvh(const ff_scene* s, void* nodes, uint64_t nodes_capacity, void* tris,
                            uint64_t tris_capacity, uint32_t* num_nodes, uint32_t* num_tris)
{
    if (!s) return FF_ERR_INVALID_ARG;
    ff_context* ctx = s->ctx;
    return guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        if (num_nodes) *num_nodes = s->num_nodes;
        if (num_tris) *num_tris = s->num_tris;
        const uint64_t nb = (uint64_t)sizeof(FFNode8) * s->num_nodes, tb = (uint64_t)sizeof(FFTri) * s->num_tris;
        FF_REQUIRE(!nodes || nodes_capacity >= nb, "node buffer smaller than num_nodes * 80 bytes");
        FF_REQUIRE(!tris || tris_capacity >= tb, "triangle buffer smaller than num_tris * 48 bytes");
        if (nodes && nb) FF_CUDA_CHECK(cudaMemcpyAsync(nodes, s->nodes.ptr, nb, cudaMemcpyDeviceToHost, ctx->stream));
        if (tris && tb) FF_CUDA_CHECK(cudaMemcpyAsync(tris, s->tris.ptr, tb, cudaMemcpyDeviceToHost, ctx->stream));
        FF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

namespace {

// Rays per chunk of a host-pointer trace: 64 MB in, 32 MB out.
constexpr uint64_t kIoChunk = 1ull << 21;

// The host-pointer trace as a three-stage pipeline over chunks: the copy in
// of chunk i + 1 (io_in) and the copy out of chunk i - 1 (io_out) run beside
// the trace of chunk i (the context's stream), so both copy directions are
// busy at once and the call takes about the longer of the two copies instead
// of their sum.  Every chunk has its own range of the staging buffers; one
// event per edge suffices because each wait is enqueued right after the
// record it waits for.  Returns with all three streams' work enqueued; the
// caller synchronises.
void trace_host_chunks(ff_context* ctx, const ff_scene* s, const ff_ray* rays, uint64_t n, ff_hit* hits, bool any,
                       bool two)
{
    if (!ctx->io_in) {
        FF_CUDA_CHECK(cudaStreamCreateWithFlags(&ctx->io_in, cudaStreamNonBlocking));
        FF_CUDA_CHECK(cudaStreamCreateWithFlags(&ctx->io_out, cudaStreamNonBlocking));
        FF_CUDA_CHECK(cudaEventCreateWithFlags(&ctx->io_ev_start, cudaEventDisableTiming));
        FF_CUDA_CHECK(cudaEventCreateWithFlags(&ctx->io_ev_in, cudaEventDisableTiming));
        FF_CUDA_CHECK(cudaEventCreateWithFlags(&ctx->io_ev_traced, cudaEventDisableTiming));
    }
    ff_ray* d_rays = ctx->io_rays.as<ff_ray>();
    ff_hit* d_hits = ctx->io_hits.as<ff_hit>();
    try {
        // the copies in start after the work already on the context's stream
        FF_CUDA_CHECK(cudaEventRecord(ctx->io_ev_start, ctx->stream));
        FF_CUDA_CHECK(cudaStreamWaitEvent(ctx->io_in, ctx->io_ev_start, 0));
        for (uint64_t off = 0; off < n; off += kIoChunk) {
            const uint64_t m = std::min(kIoChunk, n - off);
            FF_CUDA_CHECK(cudaMemcpyAsync(d_rays + off, rays + off, sizeof(ff_ray) * m, cudaMemcpyHostToDevice,
                                          ctx->io_in));
            FF_CUDA_CHECK(cudaEventRecord(ctx->io_ev_in, ctx->io_in));
            FF_CUDA_CHECK(cudaStreamWaitEvent(ctx->stream, ctx->io_ev_in, 0));
            ff_launch_trace(ctx, s, d_rays + off, m, d_hits + off, any, two);
            FF_CUDA_CHECK(cudaEventRecord(ctx->io_ev_traced, ctx->stream));
            FF_CUDA_CHECK(cudaStreamWaitEvent(ctx->io_out, ctx->io_ev_traced, 0));
            FF_CUDA_CHECK(cudaMemcpyAsync(hits + off, d_hits + off, sizeof(ff_hit) * m, cudaMemcpyDeviceToHost,
                                          ctx->io_out));
        }
        // the context's stream ends after the last copy out
        FF_CUDA_CHECK(cudaEventRecord(ctx->io_ev_traced, ctx->io_out));
        FF_CUDA_CHECK(cudaStreamWaitEvent(ctx->stream, ctx->io_ev_traced, 0));
    } catch (...) {
        // no copy may still touch the caller's buffers after the call returns
        cudaStreamSynchronize(ctx->io_in);
        cudaStreamSynchronize(ctx->stream);
        cudaStreamSynchronize(ctx->io_out);
        throw;
    }
}

}  // namespace

ff_status ff_trace(ff_context* ctx, const ff_scene* s, const ff_ray* rays, uint64_t n, ff_hit* hits,
                   uint32_t flags)
{
    if (!ctx || !s) return FF_ERR_INVALID_ARG;
    if (n == 0) return FF_OK;
    if (!rays || !hits) return FF_ERR_INVALID_ARG;
    if (s->ctx != ctx) {
        ctx->last_error = "scene belongs to another context";
        return FF_ERR_INVALID_ARG;
    }
    return guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        const bool any = (flags & FF_TRACE_ANY) != 0;
        const bool two = (flags & FF_TRACE_TWO_SIDED) != 0;
        FF_REQUIRE(!(any && two), "FF_TRACE_TWO_SIDED applies to closest hits (any-hit rays are two-sided already)");
        if (flags & FF_MEM_DEVICE) {
            FF_REQUIRE((reinterpret_cast<uintptr_t>(rays) & 15) == 0 && (reinterpret_cast<uintptr_t>(hits) & 15) == 0,
                       "device rays and hits must be 16-byte aligned");
            ff_launch_trace(ctx, s, rays, n, hits, any, two);
        } else {
            ctx->io_rays.alloc(sizeof(ff_ray) * n);
            ctx->io_hits.alloc(sizeof(ff_hit) * n);
            trace_host_chunks(ctx, s, rays, n, hits, any, two);
            unsigned int err = 0;
            FF_CUDA_CHECK(cudaMemcpyAsync(&err, ctx->counters.as<char>() + 8, sizeof(err), cudaMemcpyDeviceToHost,
                                          ctx->stream));
            FF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
            if (err) {
                FF_CUDA_CHECK(cudaMemsetAsync(ctx->counters.as<char>() + 8, 0, sizeof(err), ctx->stream));
                throw FFError{FF_ERR_INTERNAL, "traversal exceeded its step bound (malformed BVH)"};
            }
        }
    });
}

ff_status ff_trace_count(ff_context* ctx, const ff_scene* s, const ff_ray* rays, uint64_t n, uint32_t flags,
                         uint64_t* out)
{
    if (!ctx || !s || !out) return FF_ERR_INVALID_ARG;
    if (n && !rays) return FF_ERR_INVALID_ARG;
    if (s->ctx != ctx) {
        ctx->last_error = "scene belongs to another context";
        return FF_ERR_INVALID_ARG;
    }
    return guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        const bool any = (flags & FF_TRACE_ANY) != 0;
        const bool two = (flags & FF_TRACE_TWO_SIDED) != 0;
        FF_REQUIRE(!(any && two), "FF_TRACE_TWO_SIDED applies to closest hits");
        const ff_ray* d_rays = rays;
        if (flags & FF_MEM_DEVICE) {
            FF_REQUIRE((reinterpret_cast<uintptr_t>(rays) & 15) == 0, "device rays must be 16-byte aligned");
        } else if (n) {
            ctx->io_rays.alloc(sizeof(ff_ray) * n);
            FF_CUDA_CHECK(cudaMemcpyAsync(ctx->io_rays.ptr, rays, sizeof(ff_ray) * n, cudaMemcpyHostToDevice,
                                          ctx->stream));
            d_rays = ctx->io_rays.as<ff_ray>();
        }
        // counters: [16..31] the two work totals, [8..11] the traversal error count
        unsigned long long* d_out = reinterpret_cast<unsigned long long*>(ctx->counters.as<char>() + 16);
        unsigned int* err = reinterpret_cast<unsigned int*>(ctx->counters.as<char>() + 8);
        FF_CUDA_CHECK(cudaMemsetAsync(d_out, 0, 2 * sizeof(unsigned long long), ctx->stream));
        ff_launch_trace_count(ctx, s, d_rays, n, any, d_out, err, two);
        unsigned long long h[2] = {0, 0};
        unsigned int e = 0;
        FF_CUDA_CHECK(cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        FF_CUDA_CHECK(cudaMemcpyAsync(&e, err, sizeof(e), cudaMemcpyDeviceToHost, ctx->stream));
        FF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
        if (e) {
            FF_CUDA_CHECK(cudaMemsetAsync(err, 0, sizeof(e), ctx->stream));
            throw FFError{FF_ERR_INTERNAL, "traversal exceeded its step bound (malformed BVH)"};
        }
        out[0] = h[0];
        out[1] = h[1];
        out[2] = sizeof(FFNode8);
        out[3] = sizeof(FFTri);
    });
}

}  // extern "C"

extern "C" ff_status ff_render(ff_context* ctx, ff_scene* scene, const ff_render_settings* settings, ff_film* film,
                               ff_render_stats* stats)
{
    if (!ctx || !scene || !settings || !film) return FF_ERR_INVALID_ARG;
    if (scene->ctx != ctx || film->ctx != ctx) {
        ctx->last_error = "scene or film belongs to another context";
        return FF_ERR_INVALID_ARG;
    }
    return guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        ff_wavefront_render(ctx, scene, settings, film, stats);
    });
}

extern "C" ff_status ff_render_adjoint(ff_context* ctx, ff_scene* scene, const ff_render_settings* settings,
                                       const ff_adjoint_desc* desc, ff_render_stats* stats)
{
    if (!ctx || !scene || !settings || !desc) return FF_ERR_INVALID_ARG;
    if (scene->ctx != ctx) {
        ctx->last_error = "scene belongs to another context";
        return FF_ERR_INVALID_ARG;
    }
    return guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        FF_REQUIRE(settings->mode == FF_MODE_CORRECTED, "the adjoint follows FF_MODE_CORRECTED paths");
        if (stats) std::memset(stats, 0, sizeof(*stats));
        ff_adjoint_render(ctx, scene, settings, desc, stats);
    });
}

extern "C" ff_status ff_scene_set_texture(ff_scene* s, uint32_t index, const float* rgb, uint32_t flags)
{
    if (!s || !rgb) return FF_ERR_INVALID_ARG;
    ff_context* ctx = s->ctx;
    return guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        FF_REQUIRE(index < s->textures.size(), "texture index out of range");
        DevBuf* b = s->textures[index];
        FF_CUDA_CHECK(cudaMemcpyAsync(b->ptr, rgb, b->bytes,
                                      (flags & FF_MEM_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                      ctx->stream));
        FF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

extern "C" ff_status ff_scene_set_environment(ff_scene* s, const float* rgb, uint32_t flags)
{
    if (!s || !rgb) return FF_ERR_INVALID_ARG;
    ff_context* ctx = s->ctx;
    return guarded(ctx, [&] {
        DeviceGuard g(ctx->device);
        FF_REQUIRE(s->env.width > 0, "scene has no environment map");
        FF_CUDA_CHECK(cudaMemcpyAsync(s->env.rgb.ptr, rgb, sizeof(float3) * s->env.width * s->env.height,
                                      (flags & FF_MEM_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                      ctx->stream));
        if (!(flags & FF_ENV_KEEP_TABLES)) ff_build_env_tables(ctx, s);
        else ff_env_pack(ctx, s);
        FF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

// ------------------------------------------------------------- test hooks

FFAllocStats g_ff_alloc;

extern "C" ff_status ff_debug_alloc_stats(uint64_t* total, int64_t* live)
{
    if (total) *total = g_ff_alloc.total.load();
    if (live) *live = g_ff_alloc.live.load();
    return FF_OK;
}

extern "C" ff_status ff_debug_fail_alloc_after(int64_t n)
{
    g_ff_alloc.fail_after.store(n < 0 ? -1 : n);
    return FF_OK;
}
