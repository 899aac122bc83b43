// ff_envmap.cu — environment-map importance tables built by device scans.
//
// Replaces g_compute_pdf_denom, g_compute_marginal_dist,
// g_compute_conditional_dist and g_write_pdf_texture
// (CUDA-RayTracer/kernel.cu:65-149), which run as single-thread <<<1,1>>>
// loops (and one thread per row) over every texel.  Same tables, same FP64
// accumulation and the same luminance of the bilinear fetch at each texel's
// corner (u = i/w, v = j/h); the sums over whole rows are reassociated into
// block reductions, while the CDFs are the reference's running sums (one
// thread along each row, and along the marginal), so that every CDF is sorted
// by construction (a scan's tree of partial sums can leave two neighbours one
// ulp out of order):
//   k_env_rows      one block per row: luminance of every texel, row sum
//   k_env_marginal  one block: pdf denominator, marginal pdf and CDF
//   k_env_cond      one block per row: the pdf texture lum * sin(pi v) /
//                   denom * w*h / (2 pi^2) (all threads) and the conditional
//                   CDF (one running sum)
//   k_env_guide     one block per CDF: the guide table of its searches
//                   (kGuideFull, ff_shade.cuh)
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
    __shared__ union {
        typename Reduce::TempStorage r;
    } tmp;
    __shared__ double s_denom;
    // pdf denominator: sum_j sum_i lum_ij * sin(pi v_j)
    double acc = 0.0;
    for (int j = threadIdx.x; j < h; j += kEnvBlock) acc += row_sum[j] * row_sin(j, h);
    const double d = Reduce(tmp.r).Sum(acc);
    if (threadIdx.x == 0) s_denom = d;
    __syncthreads();
    const double dn = s_denom;
    // marginal pdf, then its CDF as the reference sums it:
    // marginal_y[j] = marginal_p[j] + marginal_y[j - 1]
    for (int j = threadIdx.x; j < h; j += kEnvBlock) marginal_p[j] = row_sum[j] * (row_sin(j, h) / dn);
    __syncthreads();
    if (threadIdx.x == 0) {
        double run = 0.0;
        for (int j = 0; j < h; ++j) {
            run = j == 0 ? marginal_p[0] : marginal_p[j] + run;
            marginal_y[j] = run;
        }
        *denom = dn;
    }
}

__global__ void __launch_bounds__(kEnvBlock) k_env_cond(const float* __restrict__ lum, int w, int h,
                                                        const double* __restrict__ marginal_p,
                                                        const double* __restrict__ denom, double* __restrict__ cond,
                                                        float* __restrict__ pdf)
{
    const int j = blockIdx.x;
    const double s = row_sin(j, h);
    const double dn = *denom;
    const double val = s / (dn * marginal_p[j]);
    const float scale = (float)(w * h) / (2.f * FF_PI * FF_PI);
    const float* row = lum + (size_t)j * w;
    for (int i = threadIdx.x; i < w; i += kEnvBlock) {
        float p = (float)(((double)row[i] * s) / dn);
        pdf[(size_t)j * w + i] = p * scale;
    }
    // conds_y[y][x] = lum * val + conds_y[y][x - 1]: one dependent add per
    // texel (about 2,000 per row), rows in parallel
    if (threadIdx.x == 0) {
        double run = 0.0;
        double* c = cond + (size_t)j * w;
        for (int i = 0; i < w; ++i) {
            const double t = (double)row[i] * val;
            run = i == 0 ? t : t + run;
            c[i] = run;
        }
    }
}

// One block per CDF: blockIdx.x < h is conditional row blockIdx.x, h the
// marginal.  Entry k of its guide = upper_bound of k / G, by the search loop
// of upper_bound_ref; every entry kGuideFull when the list is not sorted.
__global__ void __launch_bounds__(kEnvBlock) k_env_guide(const double* __restrict__ marginal,
                                                         const double* __restrict__ cond, int w, int h,
                                                         uint32_t* __restrict__ guide_m, uint32_t* __restrict__ guide_c)
{
    const int j = blockIdx.x;
    const bool is_row = j < h;
    const double* list = is_row ? cond + (size_t)j * w : marginal;
    const int size = is_row ? w : h;
    const int G = is_row ? kGuideCond : kGuideMarginal;
    uint32_t* g = is_row ? guide_c + (size_t)j * (kGuideCond + 1) : guide_m;
    int bad = 0;
    for (int i = threadIdx.x; i < size; i += kEnvBlock)
        bad |= (i + 1 < size) ? !(list[i] <= list[i + 1]) : !(list[i] == list[i]);
    bad = __syncthreads_or(bad);
    for (int k = threadIdx.x; k <= G; k += kEnvBlock) {
        if (bad) {
            g[k] = kGuideFull;
            continue;
        }
        const float val = (float)k / (float)G;
        int left = 0, right = size;
        while (left < right) {
            const int middle = (right - left) / 2 + left;
            if ((double)val >= list[middle]) left = middle + 1;
            else right = middle;
        }
        g[k] = (uint32_t)left;
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
    e.guide.alloc(sizeof(uint32_t) * ((size_t)kGuideMarginal + 1 + (size_t)h * (kGuideCond + 1)));
    k_env_guide<<<h + 1, kEnvBlock, 0, st>>>(e.marginal.as<double>(), e.conditional.as<double>(), w, h,
                                             e.guide.as<uint32_t>(), e.guide.as<uint32_t>() + kGuideMarginal + 1);
    FF_CUDA_CHECK(cudaGetLastError());
    ff_env_pack(ctx, s);
    FF_CUDA_CHECK(cudaStreamSynchronize(st));
}

namespace {

__global__ void k_env_pick(FFEnvView e, const float2* __restrict__ exy, uint64_t n, int2* __restrict__ xy)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float ex = exy[i].x, ey = exy[i].y;
    // the searches and clamps of env_sample / env_sample_corrected
    int y = (int)((float)upper_bound_ref<kGuideMarginal>(e.marginal, e.height, ey, e.guide_m) - 1.f);
    y = y < 0 ? 0 : (y >= e.height ? e.height - 1 : y);
    int x = (int)((float)upper_bound_ref<kGuideCond>(e.cond + (size_t)y * e.width, e.width, ex, guide_row(e, y)) - 1.f);
    x = x < 0 ? 0 : (x >= e.width ? e.width - 1 : x);
    xy[i] = make_int2(x, y);
}

}  // namespace

extern "C" ff_status ff_debug_env_pick(const ff_scene* scene, const float* exy, uint64_t n, int32_t* xy)
{
    if (!scene || (n && (!exy || !xy))) return FF_ERR_INVALID_ARG;
    ff_context* ctx = scene->ctx;
    if (scene->env.width == 0) {
        ctx->last_error = "scene has no environment map";
        return FF_ERR_INVALID_ARG;
    }
    if (n == 0) return FF_OK;
    if (n > (1ull << 32)) {
        ctx->last_error = "ff_debug_env_pick: more than 2^32 draws";
        return FF_ERR_INVALID_ARG;
    }
    try {
        FF_CUDA_CHECK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        DevBuf d_in, d_out;
        d_in.alloc(sizeof(float2) * n);
        d_out.alloc(sizeof(int2) * n);
        FF_CUDA_CHECK(cudaMemcpyAsync(d_in.ptr, exy, sizeof(float2) * n, cudaMemcpyHostToDevice, st));
        k_env_pick<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ff_env_view(scene), d_in.as<float2>(), n,
                                                                 d_out.as<int2>());
        FF_CUDA_CHECK(cudaGetLastError());
        FF_CUDA_CHECK(cudaMemcpyAsync(xy, d_out.ptr, sizeof(int2) * n, cudaMemcpyDeviceToHost, st));
        FF_CUDA_CHECK(cudaStreamSynchronize(st));
        return FF_OK;
    } catch (const FFError& err) {
        ctx->last_error = err.msg;
        return err.status;
    }
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
