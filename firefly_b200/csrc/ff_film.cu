// ff_film.cu — headless film: FP32 radiance sums with Kahan compensation and
// per-pixel sample counts.
//
// Replaces the reference's accumulatebuffer / n_samples pair
// (CUDA-RayTracer/PathTracer.cpp:22-23, cleared at :150-170) and the char4
// surface written by wf_logic (kernel.cu:447-454) through GL interop.
#include <new>

#include "ff_internal.h"

namespace {

__global__ void k_tonemap(const float4* __restrict__ acc, const float4* __restrict__ comp,
                          const uint32_t* __restrict__ cnt, uint32_t n, float exposure, uchar4* __restrict__ out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // kernel.cu:447-452: accum / n * exposure, then x / (1 + x), then (int)255 * c
    uint32_t k = cnt[i];
    float4 a = acc[i];
    float4 c = comp[i];
    float3 s = make_float3(a.x - c.x, a.y - c.y, a.z - c.z);
    uchar4 o = make_uchar4(0, 0, 0, 255);
    if (k >= 1) {
        float inv = (float)k;
        float3 col = make_float3(s.x / inv * exposure, s.y / inv * exposure, s.z / inv * exposure);
        col = make_float3(col.x / (col.x + 1.f), col.y / (col.y + 1.f), col.z / (col.z + 1.f));
        // the reference stores (int)255 * c into a signed char4; values above
        // 127 wrap there.  The headless film saturates to 0..255 instead.
        o = make_uchar4((unsigned char)fminf(fmaxf(255.f * col.x, 0.f), 255.f),
                        (unsigned char)fminf(fmaxf(255.f * col.y, 0.f), 255.f),
                        (unsigned char)fminf(fmaxf(255.f * col.z, 0.f), 255.f), 255);
    }
    out[i] = o;
}

__global__ void k_resolve(const float4* __restrict__ acc, const float4* __restrict__ comp, uint32_t n,
                          float4* __restrict__ out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = acc[i], c = comp[i];
    out[i] = make_float4(a.x - c.x, a.y - c.y, a.z - c.z, 0.f);
}

template <class F>
ff_status film_guard(ff_film* f, F&& fn)
{
    try {
        fn();
        return FF_OK;
    } catch (const FFError& e) {
        f->ctx->last_error = e.msg;
        return e.status;
    } catch (...) {
        f->ctx->last_error = "unknown internal error";
        return FF_ERR_INTERNAL;
    }
}

}  // namespace

extern "C" {

ff_status ff_film_create(ff_context* ctx, uint32_t w, uint32_t h, ff_film** out)
{
    if (!ctx || !out || w == 0 || h == 0) return FF_ERR_INVALID_ARG;
    if ((uint64_t)w * h > (1ull << 30)) {
        ctx->last_error = "film too large";
        return FF_ERR_INVALID_ARG;
    }
    ff_film* f = new (std::nothrow) ff_film();
    if (!f) return FF_ERR_OOM;
    f->ctx = ctx;
    f->width = w;
    f->height = h;
    ff_status st = film_guard(f, [&] {
        FF_CUDA_CHECK(cudaSetDevice(ctx->device));
        const size_t n = (size_t)w * h;
        f->accum.alloc(sizeof(float4) * n);
        f->comp.alloc(sizeof(float4) * n);
        f->count.alloc(sizeof(uint32_t) * n);
        f->staging.alloc(sizeof(float4) * n);
        FF_CUDA_CHECK(cudaMemsetAsync(f->accum.ptr, 0, sizeof(float4) * n, ctx->stream));
        FF_CUDA_CHECK(cudaMemsetAsync(f->comp.ptr, 0, sizeof(float4) * n, ctx->stream));
        FF_CUDA_CHECK(cudaMemsetAsync(f->count.ptr, 0, sizeof(uint32_t) * n, ctx->stream));
        FF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
    if (st != FF_OK) {
        delete f;
        return st;
    }
    *out = f;
    return FF_OK;
}

ff_status ff_film_destroy(ff_film* f)
{
    if (!f) return FF_ERR_INVALID_ARG;
    cudaSetDevice(f->ctx->device);
    cudaStreamSynchronize(f->ctx->stream);
    delete f;
    return FF_OK;
}

ff_status ff_film_clear(ff_film* f)
{
    if (!f) return FF_ERR_INVALID_ARG;
    return film_guard(f, [&] {
        const size_t n = (size_t)f->width * f->height;
        cudaStream_t st = f->ctx->stream;
        FF_CUDA_CHECK(cudaMemsetAsync(f->accum.ptr, 0, sizeof(float4) * n, st));
        FF_CUDA_CHECK(cudaMemsetAsync(f->comp.ptr, 0, sizeof(float4) * n, st));
        FF_CUDA_CHECK(cudaMemsetAsync(f->count.ptr, 0, sizeof(uint32_t) * n, st));
    });
}

ff_status ff_film_read(ff_film* f, float* rgba, uint32_t* n_samples, uint32_t flags)
{
    if (!f) return FF_ERR_INVALID_ARG;
    return film_guard(f, [&] {
        const size_t n = (size_t)f->width * f->height;
        cudaStream_t st = f->ctx->stream;
        const bool dev = (flags & FF_MEM_DEVICE) != 0;
        if (rgba) {
            float4* dst = dev ? reinterpret_cast<float4*>(rgba) : f->staging.as<float4>();
            k_resolve<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(f->accum.as<float4>(), f->comp.as<float4>(),
                                                                   (uint32_t)n, dst);
            FF_CUDA_CHECK(cudaGetLastError());
            if (!dev) {
                FF_CUDA_CHECK(cudaMemcpyAsync(rgba, dst, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
                FF_CUDA_CHECK(cudaStreamSynchronize(st));
            }
        }
        if (n_samples) {
            FF_CUDA_CHECK(cudaMemcpyAsync(n_samples, f->count.ptr, sizeof(uint32_t) * n,
                                          dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
        }
        if (!dev) FF_CUDA_CHECK(cudaStreamSynchronize(st));
    });
}

ff_status ff_film_tonemap(ff_film* f, float exposure, uint8_t* rgba8, uint32_t flags)
{
    if (!f || !rgba8) return FF_ERR_INVALID_ARG;
    return film_guard(f, [&] {
        const size_t n = (size_t)f->width * f->height;
        cudaStream_t st = f->ctx->stream;
        const bool dev = (flags & FF_MEM_DEVICE) != 0;
        uchar4* dst = dev ? reinterpret_cast<uchar4*>(rgba8) : f->staging.as<uchar4>();
        k_tonemap<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(f->accum.as<float4>(), f->comp.as<float4>(),
                                                               f->count.as<uint32_t>(), (uint32_t)n, exposure, dst);
        FF_CUDA_CHECK(cudaGetLastError());
        if (!dev) {
            FF_CUDA_CHECK(cudaMemcpyAsync(rgba8, dst, sizeof(uchar4) * n, cudaMemcpyDeviceToHost, st));
            FF_CUDA_CHECK(cudaStreamSynchronize(st));
        }
    });
}

}  // extern "C"
