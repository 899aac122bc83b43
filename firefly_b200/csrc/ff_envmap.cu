// ff_envmap.cu — environment-map importance tables built by device scans.
//
// Replaces g_compute_pdf_denom, g_compute_marginal_dist,
// g_compute_conditional_dist and g_write_pdf_texture
// (CUDA-RayTracer/kernel.cu:65-149), which run as single-thread <<<1,1>>>
// loops (and one thread per row) over every texel.  Same tables, same FP64
// accumulation and the same luminance of the bilinear fetch at each texel's
// corner (u = i/w, v = j/h); the sums are reassociated into per-row block
// reductions and block scans:
//   k_env_rows      one block per row: luminance of every texel, row sum
//   k_env_marginal  one block: pdf denominator, marginal pdf and CDF (scan)
//   k_env_cond      one block per row: conditional CDF (block scan) and the
//                   pdf texture lum * sin(pi v) / denom * w*h / (2 pi^2)
// Traffic per texel: 12 B of RGB read (L2-resident neighbours for the
// bilinear weights), 4 B luminance written and read back, 8 B CDF and 4 B pdf
// written: HBM-bound at about 28 B per texel.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "ff_internal.h"
#include "ff_shade.cuh"

namespace {

constexpr int kEnvBlock = 256;

__device__ __forceinline__ double row_sin(int j, int h)
{
    // sin(M_PI * v) with M_PI a float constant: the float sine of a float
    // argument, widened.  The reference's host build gets a correctly rounded
    // sinf from libm; the double sine rounded to float reproduces it (the
    // device's single-precision sinf may differ in the last bit).
    const float v = (float)j / (float)h;
    return (double)(float)sin((double)(FF_PI * v));
}

__global__ void __launch_bounds__(kEnvBlock) k_env_rows(const float3* __restrict__ rgb, int w, int h,
                                                        float* __restrict__ lum, double* __restrict__ row_sum)
{
    using Reduce = cub::BlockReduce<double, kEnvBlock>;
    __shared__ typename Reduce::TempStorage tmp;
    const int j = blockIdx.x;
    const float v = (float)j / (float)h;
    double acc = 0.0;
    for (int i = threadIdx.x; i < w; i += kEnvBlock) {
        const float u = (float)i / (float)w;
        const float l = luminance(tex_bilinear(rgb, w, h, u, v));
        lum[(size_t)j * w + i] = l;
        acc += (double)l;
    }
    const double total = Reduce(tmp).Sum(acc);
    if (threadIdx.x == 0) row_sum[j] = total;
}

__global__ void __launch_bounds__(kEnvBlock) k_env_marginal(const double* __restrict__ row_sum, int h,
                                                            double* __restrict__ marginal_p,
                                                            double* __restrict__ marginal_y, double* __restrict__ denom)
{
    using Reduce = cub::BlockReduce<double, kEnvBlock>;
    using Scan = cub::BlockScan<double, kEnvBlock>;
    __shared__ union {
        typename Reduce::TempStorage r;
        typename Scan::TempStorage s;
    } tmp;
    __shared__ double s_denom;
    // pdf denominator: sum_j sum_i lum_ij * sin(pi v_j)
    double acc = 0.0;
    for (int j = threadIdx.x; j < h; j += kEnvBlock) acc += row_sum[j] * row_sin(j, h);
    const double d = Reduce(tmp.r).Sum(acc);
    if (threadIdx.x == 0) s_denom = d;
    __syncthreads();
    const double dn = s_denom;
    // marginal pdf and its inclusive scan, in chunks of kEnvBlock rows
    double carry = 0.0;
    for (int base = 0; base < h; base += kEnvBlock) {
        const int j = base + threadIdx.x;
        double mp = 0.0;
        if (j < h) {
            mp = row_sum[j] * (row_sin(j, h) / dn);
            marginal_p[j] = mp;
        }
        double incl;
        double chunk_total;
        Scan(tmp.s).InclusiveSum(mp, incl, chunk_total);
        if (j < h) marginal_y[j] = carry + incl;
        carry += chunk_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *denom = dn;
}

__global__ void __launch_bounds__(kEnvBlock) k_env_cond(const float* __restrict__ lum, int w, int h,
                                                        const double* __restrict__ marginal_p,
                                                        const double* __restrict__ denom, double* __restrict__ cond,
                                                        float* __restrict__ pdf)
{
    using Scan = cub::BlockScan<double, kEnvBlock>;
    __shared__ typename Scan::TempStorage tmp;
    const int j = blockIdx.x;
    const double s = row_sin(j, h);
    const double dn = *denom;
    const double val = s / (dn * marginal_p[j]);
    const float scale = (float)(w * h) / (2.f * FF_PI * FF_PI);
    // each thread owns one contiguous chunk of the row
    const int chunk = (w + kEnvBlock - 1) / kEnvBlock;
    const int i0 = min(w, (int)threadIdx.x * chunk), i1 = min(w, i0 + chunk);
    const float* row = lum + (size_t)j * w;
    double local = 0.0;
    for (int i = i0; i < i1; ++i) local += (double)row[i] * val;
    double prefix;
    Scan(tmp).ExclusiveSum(local, prefix);
    double run = prefix;
    for (int i = i0; i < i1; ++i) {
        const double l = (double)row[i];
        run += l * val;
        cond[(size_t)j * w + i] = run;
        float p = (float)((l * s) / dn);
        pdf[(size_t)j * w + i] = p * scale;
    }
}

// (r, g, b, pdf) per texel for the path kernels (FFEnvView::texel4).
__global__ void k_env_pack(const float3* __restrict__ rgb, const float* __restrict__ pdf, size_t n,
                           float4* __restrict__ out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 c = rgb[i];
    out[i] = make_float4(c.x, c.y, c.z, pdf[i]);
}

}  // namespace

// Repack after the texels or the pdf changed (ff_scene_set_environment keeps
// the tables when asked to: the new texels with the old pdf).
void ff_env_pack(ff_context* ctx, ff_scene* s)
{
    FFEnvLight& e = s->env;
    const size_t n = (size_t)e.width * e.height;
    if (!n || !e.pdf.ptr) return;
    e.texel4.alloc(sizeof(float4) * n);
    k_env_pack<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(e.rgb.as<float3>(), e.pdf.as<float>(), n,
                                                                     e.texel4.as<float4>());
    FF_CUDA_CHECK(cudaGetLastError());
}

void ff_build_env_tables(ff_context* ctx, ff_scene* s)
{
    FFEnvLight& e = s->env;
    const int w = e.width, h = e.height;
    cudaStream_t st = ctx->stream;
    e.marginal.alloc(sizeof(double) * h);
    e.conditional.alloc(sizeof(double) * (size_t)w * h);
    e.pdf.alloc(sizeof(float) * (size_t)w * h);
    e.denom.alloc(sizeof(double) * 2);
    DevBuf lum, rows, mp;
    lum.alloc(sizeof(float) * (size_t)w * h);
    rows.alloc(sizeof(double) * h);
    mp.alloc(sizeof(double) * h);
    k_env_rows<<<h, kEnvBlock, 0, st>>>(e.rgb.as<float3>(), w, h, lum.as<float>(), rows.as<double>());
    k_env_marginal<<<1, kEnvBlock, 0, st>>>(rows.as<double>(), h, mp.as<double>(), e.marginal.as<double>(),
                                            e.denom.as<double>());
    k_env_cond<<<h, kEnvBlock, 0, st>>>(lum.as<float>(), w, h, mp.as<double>(), e.denom.as<double>(),
                                        e.conditional.as<double>(), e.pdf.as<float>());
    FF_CUDA_CHECK(cudaGetLastError());
    ff_env_pack(ctx, s);
    FF_CUDA_CHECK(cudaStreamSynchronize(st));
}

extern "C" ff_status ff_scene_read_env_tables(const ff_scene* scene, double* marginal, double* conditional, float* pdf,
                                              double* pdf_denom)
{
    if (!scene) return FF_ERR_INVALID_ARG;
    ff_context* ctx = scene->ctx;
    const FFEnvLight& e = scene->env;
    if (e.width == 0) {
        ctx->last_error = "scene has no environment map";
        return FF_ERR_INVALID_ARG;
    }
    try {
        FF_CUDA_CHECK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const size_t n = (size_t)e.width * e.height;
        if (marginal)
            FF_CUDA_CHECK(cudaMemcpyAsync(marginal, e.marginal.ptr, sizeof(double) * e.height, cudaMemcpyDeviceToHost, st));
        if (conditional)
            FF_CUDA_CHECK(cudaMemcpyAsync(conditional, e.conditional.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        if (pdf) FF_CUDA_CHECK(cudaMemcpyAsync(pdf, e.pdf.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        if (pdf_denom) FF_CUDA_CHECK(cudaMemcpyAsync(pdf_denom, e.denom.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
        FF_CUDA_CHECK(cudaStreamSynchronize(st));
        return FF_OK;
    } catch (const FFError& err) {
        ctx->last_error = err.msg;
        return err.status;
    }
}
