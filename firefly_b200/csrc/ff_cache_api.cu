// ff_cache_api.cu — extern "C" entry points of the learned radiance cache.
#include <cstring>
#include <new>

#include "ff_internal.h"

namespace {

template <class F>
ff_status cache_guard(ff_context* ctx, F&& f)
{
    try {
        int prev = -1;
        cudaGetDevice(&prev);
        if (prev != ctx->device) FF_CUDA_CHECK(cudaSetDevice(ctx->device));
        f();
        if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
        return FF_OK;
    } catch (const FFError& e) {
        ctx->last_error = e.msg;
        return e.status;
    } catch (const std::bad_alloc&) {
        ctx->last_error = "host allocation failed";
        return FF_ERR_OOM;
    } catch (...) {
        ctx->last_error = "unknown internal error";
        return FF_ERR_INTERNAL;
    }
}

size_t grid_entries(const ff_cache* c) { return (size_t)FF_CACHE_LEVELS << c->prm.log2_table_size; }

void check_err(ff_cache* c)
{
    unsigned int e = 0;
    FF_CUDA_CHECK(cudaMemcpyAsync(&e, c->err.ptr, sizeof(e), cudaMemcpyDeviceToHost, c->ctx->stream));
    FF_CUDA_CHECK(cudaStreamSynchronize(c->ctx->stream));
    if (e) {
        FF_CUDA_CHECK(cudaMemsetAsync(c->err.ptr, 0, sizeof(unsigned int), c->ctx->stream));
        throw FFError{FF_ERR_TIMEOUT, "tensor-core wait gave up in the radiance cache"};
    }
}

// Records from host or device memory, on the device.
const void* device_records(ff_cache* c, const ff_cache_record* recs, uint32_t n, uint32_t flags)
{
    if (flags & FF_MEM_DEVICE) return recs;
    c->io_recs.alloc(sizeof(ff_cache_record) * (size_t)n);
    FF_CUDA_CHECK(cudaMemcpyAsync(c->io_recs.ptr, recs, sizeof(ff_cache_record) * (size_t)n, cudaMemcpyHostToDevice,
                                  c->ctx->stream));
    return c->io_recs.ptr;
}

}  // namespace

static_assert(sizeof(ff_cache_record) == sizeof(ffc::Record), "ff_cache_record mirrors the device record");

extern "C" {

ff_status ff_cache_create(ff_context* ctx, const ff_scene* scene, const ff_cache_params* params, ff_cache** out)
{
    if (!ctx || !scene || !params || !out) return FF_ERR_INVALID_ARG;
    *out = nullptr;
    if (scene->ctx != ctx) {
        ctx->last_error = "scene belongs to another context";
        return FF_ERR_INVALID_ARG;
    }
    ff_cache* c = new (std::nothrow) ff_cache();
    if (!c) return FF_ERR_OOM;
    c->ctx = ctx;
    c->prm = *params;
    ff_status st = cache_guard(ctx, [&] {
        const ff_cache_params& p = c->prm;
        FF_REQUIRE(p.log2_table_size >= 10 && p.log2_table_size <= 24, "log2_table_size must be in [10, 24]");
        FF_REQUIRE(p.base_resolution >= 2 && p.max_resolution >= p.base_resolution && p.max_resolution <= (1u << 20),
                   "resolutions must satisfy 2 <= base <= max <= 2^20");
        FF_REQUIRE(p.lr > 0.f && p.beta1 >= 0.f && p.beta1 < 1.f && p.beta2 >= 0.f && p.beta2 < 1.f && p.eps > 0.f,
                   "invalid Adam parameters");
        int major = 0;
        FF_CUDA_CHECK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, ctx->device));
        if (major != 10) throw FFError{FF_ERR_UNSUPPORTED, "the radiance cache needs an sm_100 tensor core"};
        // the scene box, grown by 1% so that surfaces on it stay inside
        float3 lo = scene->lo, hi = scene->hi;
        const float3 e = make_float3((hi.x - lo.x) * 0.01f + 1e-4f, (hi.y - lo.y) * 0.01f + 1e-4f,
                                     (hi.z - lo.z) * 0.01f + 1e-4f);
        c->lo = make_float3(lo.x - e.x, lo.y - e.y, lo.z - e.z);
        c->hi = make_float3(hi.x + e.x, hi.y + e.y, hi.z + e.z);
        const size_t n = grid_entries(c);
        c->table.alloc(sizeof(float2) * n);
        c->table_h.alloc(sizeof(uint32_t) * n);
        c->grid_grad.alloc(sizeof(float2) * n);
        c->grid_m.alloc(sizeof(float2) * n);
        c->grid_v.alloc(sizeof(float2) * n);
        const size_t np = ff_cache_num_params();
        c->mlp.alloc(sizeof(float) * np);
        c->mlp_img.alloc(sizeof(uint16_t) * np);
        c->mlp_grad.alloc(sizeof(float) * np);
        c->mlp_m.alloc(sizeof(float) * np);
        c->mlp_v.alloc(sizeof(float) * np);
        c->loss.alloc(sizeof(float));
        c->err.alloc(sizeof(unsigned int));
        FF_CUDA_CHECK(cudaMemsetAsync(c->loss.ptr, 0, sizeof(float), ctx->stream));
        FF_CUDA_CHECK(cudaMemsetAsync(c->err.ptr, 0, sizeof(unsigned int), ctx->stream));
        ff_cache_setup_grid(c);
        ff_cache_init_params(c);
        FF_CUDA_CHECK(cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking));
        FF_CUDA_CHECK(cudaEventCreateWithFlags(&c->ev_frame, cudaEventDisableTiming));
        FF_CUDA_CHECK(cudaEventCreateWithFlags(&c->ev_trained, cudaEventDisableTiming));
        FF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
    if (st != FF_OK) {
        delete c;
        return st;
    }
    *out = c;
    return FF_OK;
}

ff_status ff_cache_destroy(ff_cache* c)
{
    if (!c) return FF_ERR_INVALID_ARG;
    cudaSetDevice(c->ctx->device);
    cudaStreamSynchronize(c->ctx->stream);
    delete c;
    return FF_OK;
}

ff_status ff_debug_cache_wait_limit(ff_cache* c, uint32_t polls)
{
    if (!c) return FF_ERR_INVALID_ARG;
    c->wait_polls = polls;
    return FF_OK;
}

ff_status ff_cache_reset(ff_cache* c)
{
    if (!c) return FF_ERR_INVALID_ARG;
    return cache_guard(c->ctx, [&] {
        ff_cache_init_params(c);
        FF_CUDA_CHECK(cudaStreamSynchronize(c->ctx->stream));
    });
}

ff_status ff_cache_query(ff_cache* c, const ff_cache_record* recs, uint32_t n, float* rgb, uint32_t flags)
{
    if (!c || (n && (!recs || !rgb))) return FF_ERR_INVALID_ARG;
    return cache_guard(c->ctx, [&] {
        if (n == 0) return;
        const void* d_recs = device_records(c, recs, n, flags);
        float* d_out = rgb;
        if (!(flags & FF_MEM_DEVICE)) {
            c->io_out.alloc(sizeof(float) * 3 * (size_t)n);
            d_out = c->io_out.as<float>();
        }
        ff_cache_launch_infer(c, d_recs, n, nullptr, d_out, nullptr);
        if (!(flags & FF_MEM_DEVICE))
            FF_CUDA_CHECK(cudaMemcpyAsync(rgb, d_out, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToHost,
                                          c->ctx->stream));
        check_err(c);
    });
}

ff_status ff_cache_train(ff_cache* c, const ff_cache_record* recs, uint32_t n, uint32_t flags, float* loss)
{
    if (!c || (n && !recs)) return FF_ERR_INVALID_ARG;
    return cache_guard(c->ctx, [&] {
        if (n == 0) return;
        cudaStream_t st = c->ctx->stream;
        const void* d_recs = device_records(c, recs, n, flags);
        FF_CUDA_CHECK(cudaMemsetAsync(c->loss.ptr, 0, sizeof(float), st));
        ff_cache_launch_train(c, d_recs, n, (flags & FF_CACHE_GRADIENTS_ONLY) != 0);
        if (loss) {
            float s = 0.f;
            FF_CUDA_CHECK(cudaMemcpyAsync(&s, c->loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, st));
            check_err(c);
            *loss = s / (float)n;
        } else {
            check_err(c);
        }
    });
}

ff_status ff_cache_read_params(ff_cache* c, float* mlp, float* grid, float* grad_mlp, float* grad_grid)
{
    if (!c) return FF_ERR_INVALID_ARG;
    return cache_guard(c->ctx, [&] {
        cudaStream_t st = c->ctx->stream;
        const size_t np = ff_cache_num_params(), ng = grid_entries(c) * 2;
        if (mlp) FF_CUDA_CHECK(cudaMemcpyAsync(mlp, c->mlp.ptr, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
        if (grad_mlp)
            FF_CUDA_CHECK(cudaMemcpyAsync(grad_mlp, c->mlp_grad.ptr, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
        if (grid) FF_CUDA_CHECK(cudaMemcpyAsync(grid, c->table.ptr, sizeof(float) * ng, cudaMemcpyDeviceToHost, st));
        if (grad_grid)
            FF_CUDA_CHECK(cudaMemcpyAsync(grad_grid, c->grid_grad.ptr, sizeof(float) * ng, cudaMemcpyDeviceToHost, st));
        FF_CUDA_CHECK(cudaStreamSynchronize(st));
    });
}

ff_status ff_cache_write_params(ff_cache* c, const float* mlp, const float* grid)
{
    if (!c) return FF_ERR_INVALID_ARG;
    return cache_guard(c->ctx, [&] {
        cudaStream_t st = c->ctx->stream;
        const size_t np = ff_cache_num_params(), ng = grid_entries(c) * 2;
        if (mlp) FF_CUDA_CHECK(cudaMemcpyAsync(c->mlp.ptr, mlp, sizeof(float) * np, cudaMemcpyHostToDevice, st));
        if (grid) FF_CUDA_CHECK(cudaMemcpyAsync(c->table.ptr, grid, sizeof(float) * ng, cudaMemcpyHostToDevice, st));
        ff_cache_refresh_copies(c);
        FF_CUDA_CHECK(cudaStreamSynchronize(st));
    });
}

ff_status ff_render_cached(ff_context* ctx, ff_scene* scene, ff_cache* cache, const ff_render_settings* settings,
                           ff_film* film, ff_render_stats* stats)
{
    if (!ctx || !scene || !cache || !settings || !film) return FF_ERR_INVALID_ARG;
    if (scene->ctx != ctx || cache->ctx != ctx || film->ctx != ctx) {
        ctx->last_error = "scene, cache and film must belong to the context";
        return FF_ERR_INVALID_ARG;
    }
    return cache_guard(ctx, [&] {
        FF_REQUIRE(settings->mode == FF_MODE_CORRECTED, "the cached render follows FF_MODE_CORRECTED paths");
        if (stats) std::memset(stats, 0, sizeof(*stats));
        ff_cached_render(ctx, scene, cache, settings, film, stats);
        check_err(cache);
    });
}

}  // extern "C"
