// ff_cache.cu — learned radiance cache: a multiresolution hash grid and a
// 64-wide MLP (4 hidden ReLU layers, 3 outputs, no biases except through the
// constant input) evaluated and trained on the fifth-generation tensor cores.
//
// Both kernels work on tiles of 128 records with 256 threads (8 warps):
// thread (warp w, lane) owns row r = 32 (w % 4) + lane of the tile and half
// h = w / 4 of its 64 columns, which is exactly the part of a 128-lane TMEM
// accumulator its warp may read (subpartition w % 4).
//   k_cache_infer  encode -> X (smem) -> 5 MMAs chains (K = 64 in four K=16
//                  steps) with a ReLU/bf16 epilogue TMEM -> smem between
//                  layers; activations overwrite the input tile.  Its CTA
//                  runs kGroups independent tile pipelines of 4 warps (one
//                  thread per row, all 64 columns) over one copy of the
//                  weights: while one group waits on its MMAs the others
//                  gather hash-grid features, so the encoder's L2 gathers
//                  overlap the tensor-core chains of the other tiles.
//   k_cache_train  the same forward keeping every layer's activations, the
//                  relative-L2 loss gradient, then per layer (top down) the
//                  weight gradient act^T * delta (M = 64, both operands
//                  MN-major, accumulated in TMEM over all tiles of the CTA)
//                  and the input gradient delta * W (W read MN-major from
//                  the forward image); the input gradient of the hash
//                  features is scattered to the grid's FP32 gradient.
// Weights live in FP32 (master), their bf16 images pre-swizzled for shared
// memory; Adam updates both.  The grid keeps FP32 features with an FP16
// copy that the encoder reads (16 x 2^19 x 4 B = 32 MB, L2-resident).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <atomic>
#include <cmath>
#include <new>

#include "ff_cache.cuh"
#include "ff_internal.h"
#include "ff_umma.cuh"

using namespace ffc;
using namespace ffu;

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kTileBytes = 128u * 128u;             // 128 rows x 64 bf16
constexpr uint32_t kWBytes = 64u * 128u;                  // one 64 x 64 bf16 weight image
constexpr uint32_t kImgBytes = kLayers * kWBytes;         // 40 KB
constexpr uint32_t kParams = kLayers * kWidth * kWidth;   // FP32 master weights (W4 rows >= 3 stay zero)
constexpr uint32_t kWaitPolls = 1u << 22;
constexpr int kGroups = 3;                                // inference: tile pipelines per CTA
constexpr int kInferThreads = 128 * kGroups;
constexpr uint32_t kInferSmem = kImgBytes + kGroups * kTileBytes + 1024 + 64;
constexpr uint32_t kTrainSmem = kImgBytes + 6 * kTileBytes + 1024 + 64;
constexpr uint32_t kTrainTmemCols = 512;                  // D (64) + 5 weight-gradient accumulators (5 x 64)
constexpr uint32_t kInferTmemCols = 256;                 // 64 per group, allocated as a power of two

constexpr uint32_t ID_FWD = idesc_bf16(128, 64, false, false);
constexpr uint32_t ID_OUT = idesc_bf16(128, 16, false, false);
constexpr uint32_t ID_DGRAD = idesc_bf16(128, 64, false, true);
constexpr uint32_t ID_WGRAD = idesc_bf16(64, 64, true, true);

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16(uint32_t u)
{
    __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162*>(&u);
    return __bfloat1622float2(v);
}

// 8 values -> chunk c of row r of a swizzled tile
__device__ __forceinline__ void store_chunk(uint8_t* tile, uint32_t r, uint32_t c, const float* v)
{
    uint4 q = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    *reinterpret_cast<uint4*>(tile + r * 128u + (((c ^ (r & 7u)) & 7u) << 4)) = q;
}
__device__ __forceinline__ uint4 load_chunk(const uint8_t* tile, uint32_t r, uint32_t c)
{
    return *reinterpret_cast<const uint4*>(tile + r * 128u + (((c ^ (r & 7u)) & 7u) << 4));
}

// This thread's 32 inputs of row r: h = 0 -> columns 0..15 (levels 0..7) and
// 32..47 (SH); h = 1 -> columns 16..31 (levels 8..15) and 48..63.
__device__ void encode_half(const Grid& g, const Record& rec, bool valid, uint32_t h, uint32_t r, uint8_t* tile)
{
    float f[32];
    if (valid) {
        const float3 p = normalised_pos(g, rec.px, rec.py, rec.pz);
#pragma unroll   // all 8 levels' loads in flight (78 registers, no spills; query stage 2.39 -> 2.30 ms / 4 frames)
        for (int j = 0; j < 8; ++j) {
            const float2 e = level_feature(g, 8 * (int)h + j, p);
            f[2 * j] = e.x;
            f[2 * j + 1] = e.y;
        }
        if (h == 0) {
            sh16(rec.wx, rec.wy, rec.wz, f + 16);
        } else {
            f[16] = rec.nx;
            f[17] = rec.ny;
            f[18] = rec.nz;
            f[19] = rec.rough;
            f[20] = 1.f;
#pragma unroll
            for (int k = 21; k < 32; ++k) f[k] = 0.f;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 32; ++k) f[k] = 0.f;
    }
    store_chunk(tile, r, 2 * h, f);
    store_chunk(tile, r, 2 * h + 1, f + 8);
    store_chunk(tile, r, 4 + 2 * h, f + 16);
    store_chunk(tile, r, 5 + 2 * h, f + 24);
}

// ReLU epilogue: TMEM columns [32h, 32h+32) of row r -> chunks 4h..4h+3 of dst.
__device__ __forceinline__ void relu_epilogue(uint32_t taddr_row, uint32_t h, uint32_t r, uint8_t* dst)
{
    float v[32];
    tmem_ld32(taddr_row + 32u * h, v);
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = fmaxf(v[k], 0.f);
#pragma unroll
    for (int c = 0; c < 4; ++c) store_chunk(dst, r, 4 * h + c, v + 8 * c);
}

// Copy the weight images to shared memory.
__device__ __forceinline__ void load_weights(const uint4* __restrict__ img, uint8_t* w_s)
{
    uint4* d = reinterpret_cast<uint4*>(w_s);
    for (uint32_t i = threadIdx.x; i < kImgBytes / 16; i += blockDim.x) d[i] = img[i];
}

__device__ __forceinline__ void issue_forward(uint32_t d, uint32_t a_s, uint32_t w_s, uint32_t idesc)
{
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) mma_bf16(d, sw128_desc(a_s + 32u * k), sw128_desc(w_s + 32u * k), idesc, k > 0);
}

struct CacheArgs {
    Grid grid;
    const uint4* w_img;
    const Record* recs;
    const uint32_t* n_dev;      // record count on the device (or null: n)
    uint32_t offset;            // with n_dev: records before recs that are not this launch's
    uint32_t n;                 // records at most
    float* out_rgb;             // infer: n * 3 (or null)
    float4* frame;              // infer: += throughput * max(y, 0) at the record's pixel (or null)
    float* grad_w;              // train: [5][64][64]
    float* loss;                // train: sum of the per-record losses
    float inv_n;                // train: 1 / records in the batch
    unsigned int* err;
    uint32_t wait_polls;        // bound of each MMA wait (the drain after a failure keeps kWaitPolls)
};

__device__ __forceinline__ uint32_t count_of(const CacheArgs& a)
{
    if (!a.n_dev) return a.n;
    const uint32_t c = *a.n_dev;
    return c > a.offset ? min(c - a.offset, a.n) : 0u;
}

// Align the dynamic shared memory to the 1024-byte swizzle atom.
__device__ __forceinline__ uint8_t* aligned_smem(uint8_t* raw)
{
    const uint32_t s = smem_addr(raw);
    return raw + (((s + 1023u) & ~1023u) - s);
}

// Barrier of one group's 128 threads (ids 1..kGroups; 0 is __syncthreads).
__device__ __forceinline__ void group_sync(uint32_t id)
{
    asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory");
}
// The same barrier, returning whether any of the group's threads passed p.
__device__ __forceinline__ bool group_sync_or(uint32_t id, bool p)
{
    uint32_t any;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(any)
        : "r"((uint32_t)p), "r"(id)
        : "memory");
    return any != 0;
}

__global__ void __launch_bounds__(kInferThreads, 2) k_cache_infer(CacheArgs a)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = aligned_smem(smem_raw);
    uint8_t* w_s = base;
    uint64_t* mbars = reinterpret_cast<uint64_t*>(base + kImgBytes + kGroups * kTileBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbars + kGroups);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    // group g = warps 4g..4g+3; warp 4g+q reads TMEM lanes 32q.. (its subpartition)
    const uint32_t g = warp >> 2, q = warp & 3u, r = 32u * q + lane;
    uint8_t* act = base + kImgBytes + g * kTileBytes;
    const uint32_t mbar = smem_addr(mbars + g), bar = 1u + g;
    const bool leader = (tid & 127u) == 0;
    const uint32_t n = count_of(a);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    if (blockIdx.x * kGroups >= tiles) return;  // block-uniform, before any TMEM is held

    load_weights(a.w_img, w_s);
    if (tid < kGroups) mbar_init(smem_addr(mbars + tid), 1);
    __syncwarp();
    if (warp == 0) tmem_alloc(smem_addr(tslot), kInferTmemCols);
    fence_smem_async();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem_all = *tslot;
    const uint32_t tmem = tmem_all + 64u * g;   // this group's accumulator columns
    const uint32_t trow = tmem_addr(tmem, 32u * q, 0);
    const uint32_t w0 = smem_addr(w_s), x0 = smem_addr(act);
    uint32_t phase = 0;
    bool failed = false;

    for (uint32_t t = blockIdx.x * kGroups + g; t < tiles && !failed; t += gridDim.x * kGroups) {
        const uint32_t i = t * kTile + r;
        const bool valid = i < n;
        Record rec;
        if (valid) rec = a.recs[i];
        encode_half(a.grid, rec, valid, 0, r, act);
        encode_half(a.grid, rec, valid, 1, r, act);
        fence_smem_async();
        fence_before_sync();
        group_sync(bar);
        for (int l = 0; l < kLayers; ++l) {
            if (leader) {
                fence_after_sync();
                issue_forward(tmem, x0, w0 + (uint32_t)l * kWBytes, l + 1 < kLayers ? ID_FWD : ID_OUT);
                mma_commit(mbar);
            }
            const bool ok = mbar_wait(mbar, phase, a.wait_polls);
            phase ^= 1u;
            if (group_sync_or(bar, !ok)) {
                failed = true;
                break;
            }
            fence_after_sync();
            if (l + 1 < kLayers) {
                relu_epilogue(trow, 0, r, act);
                relu_epilogue(trow, 1, r, act);
            } else {
                float y[16];
                tmem_ld16(trow, y);
                if (valid) {
                    if (a.out_rgb) {
                        a.out_rgb[3 * (size_t)i + 0] = y[0];
                        a.out_rgb[3 * (size_t)i + 1] = y[1];
                        a.out_rgb[3 * (size_t)i + 2] = y[2];
                    }
                    if (a.frame) {
                        float4* f = a.frame + rec.pixel;
                        float4 c = *f;
                        c.x += rec.v0 * fmaxf(y[0], 0.f);
                        c.y += rec.v1 * fmaxf(y[1], 0.f);
                        c.z += rec.v2 * fmaxf(y[2], 0.f);
                        *f = c;
                    }
                }
            }
            fence_smem_async();
            fence_before_sync();
            group_sync(bar);
        }
    }
    if (failed && leader) {
        atomicAdd(a.err, 1u);
        mbar_wait(mbar, phase ^ 1u, kWaitPolls);   // the commit that did not arrive, once more
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem_all, kInferTmemCols);
    }
}

__global__ void __launch_bounds__(kThreads, 1) k_cache_train(CacheArgs a)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = aligned_smem(smem_raw);
    uint8_t* w_s = base;
    uint8_t* act[5];                             // X, H1..H4
    for (int l = 0; l < 5; ++l) act[l] = base + kImgBytes + (uint32_t)l * kTileBytes;
    uint8_t* dlt = base + kImgBytes + 5 * kTileBytes;
    uint64_t* mbar_p = reinterpret_cast<uint64_t*>(dlt + kTileBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(dlt + kTileBytes + 16);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t q = warp & 3u, h = warp >> 2, r = 32u * q + lane;
    const uint32_t mbar = smem_addr(mbar_p);
    const uint32_t n = count_of(a);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    if (blockIdx.x >= tiles) return;

    load_weights(a.w_img, w_s);
    if (tid == 0) mbar_init(mbar, 1);
    __syncwarp();
    if (warp == 0) tmem_alloc(smem_addr(tslot), kTrainTmemCols);
    fence_smem_async();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t trow = tmem_addr(tmem, 32u * q, 0);
    const uint32_t w0 = smem_addr(w_s), d0 = smem_addr(dlt);
    uint32_t a_s[5];
    for (int l = 0; l < 5; ++l) a_s[l] = smem_addr(act[l]);
    uint32_t phase = 0;
    bool failed = false, accumulating = false;
    float loss = 0.f;
    const float inv_n = a.n_dev ? 1.f / (float)n : a.inv_n;

    auto step = [&]() -> bool {         // commit, wait, agree
        if (tid == 0) mma_commit(mbar);
        const bool ok = mbar_wait(mbar, phase, a.wait_polls);
        phase ^= 1u;
        const bool bad = __syncthreads_or(!ok);
        fence_after_sync();
        return !bad;
    };
    auto sync_out = [&]() {             // smem writes and TMEM reads done before the next issue
        fence_smem_async();
        fence_before_sync();
        __syncthreads();
    };

    for (uint32_t t = blockIdx.x; t < tiles && !failed; t += gridDim.x) {
        const uint32_t i = t * kTile + r;
        const bool valid = i < n;
        Record rec;
        if (valid) rec = a.recs[i];
        encode_half(a.grid, rec, valid, h, r, act[0]);
        sync_out();
        // forward, keeping the activations
        for (int l = 0; l < 4 && !failed; ++l) {
            if (tid == 0) {
                fence_after_sync();
                issue_forward(tmem, a_s[l], w0 + (uint32_t)l * kWBytes, ID_FWD);
            }
            if (!step()) { failed = true; break; }
            relu_epilogue(trow, h, r, act[l + 1]);
            sync_out();
        }
        if (failed) break;
        if (tid == 0) {
            fence_after_sync();
            issue_forward(tmem, a_s[4], w0 + 4u * kWBytes, ID_OUT);
        }
        if (!step()) { failed = true; break; }
        // relative L2 loss, sum_c (y - t)^2 / (y^2 + 0.01), its gradient
        // with the denominator held constant; delta of the output layer
        if (h == 0) {
            float y[16];
            tmem_ld16(trow, y);
            float dy[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (valid) {
                const float tg[3] = {rec.v0, rec.v1, rec.v2};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float den = y[c] * y[c] + 0.01f;
                    const float e = y[c] - tg[c];
                    loss += e * e / den;
                    dy[c] = 2.f * e / den * inv_n;
                }
            }
            const float zero[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            store_chunk(dlt, r, 0, dy);
            for (uint32_t c = 1; c < 8; ++c) store_chunk(dlt, r, c, zero);
        }
        sync_out();
        // backward: layer l maps act[l] to the pre-activation whose gradient is in dlt
        for (int l = 4; l >= 0; --l) {
            if (tid == 0) {
                fence_after_sync();
                const uint32_t g = tmem + 64u + 64u * (uint32_t)l;
#pragma unroll
                for (uint32_t k = 0; k < 8; ++k)
                    mma_bf16(g, sw128_desc(a_s[l] + 2048u * k), sw128_desc(d0 + 2048u * k), ID_WGRAD,
                             (accumulating || k > 0) ? 1u : 0u);
#pragma unroll
                for (uint32_t k = 0; k < 4; ++k)
                    mma_bf16(tmem, sw128_desc(d0 + 32u * k), sw128_desc(w0 + (uint32_t)l * kWBytes + 2048u * k),
                             ID_DGRAD, k > 0);
            }
            if (!step()) { failed = true; break; }
            if (l > 0) {
                // delta of layer l: (delta W_l) * relu'(act[l])
                float v[32];
                tmem_ld32(trow + 32u * h, v);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint4 m = load_chunk(act[l], r, 4 * h + c);
                    const uint32_t mw[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float2 av = unpack_bf16(mw[j]);
                        if (!(av.x > 0.f)) v[8 * c + 2 * j] = 0.f;
                        if (!(av.y > 0.f)) v[8 * c + 2 * j + 1] = 0.f;
                    }
                    store_chunk(dlt, r, 4 * h + c, v + 8 * c);
                }
            } else {
                // input gradient of the hash features: columns 16h..16h+15 are levels 8h..8h+7
                float v[16];
                tmem_ld16(trow + 16u * h, v);
                if (valid) {
                    const float3 p = normalised_pos(a.grid, rec.px, rec.py, rec.pz);
                    for (int j = 0; j < 8; ++j) {
                        Corners c;
                        level_corners(a.grid, 8 * (int)h + j, p, c);
                        const float gx = v[2 * j], gy = v[2 * j + 1];
#pragma unroll
                        for (int k = 0; k < 8; ++k)
                            atomicAdd(a.grid.grad + c.idx[k], make_float2(c.w[k] * gx, c.w[k] * gy));
                    }
                }
            }
            sync_out();
        }
        accumulating = true;
    }
    if (!failed && accumulating) {
        // weight gradients: accumulator l holds act[l]^T delta, rows m = input
        // unit (M = 64: TMEM lanes 0-15 of each subpartition), columns n
        for (int l = 0; l < kLayers; ++l) {
            float v[32];
            tmem_ld32(trow + 64u + 64u * (uint32_t)l + 32u * h, v);
            if (lane < 16) {
                const uint32_t m = 16u * q + lane;
                float* gw = a.grad_w + (size_t)l * kWidth * kWidth;
                for (int j = 0; j < 32; ++j) {
                    const uint32_t nn = 32u * h + (uint32_t)j;
                    if (l == kLayers - 1 && nn >= (uint32_t)kOutputs) break;
                    atomicAdd(gw + nn * kWidth + m, v[j]);
                }
            }
        }
    }
    for (int off = 16; off; off >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, off);
    if (lane == 0 && loss != 0.f) atomicAdd(a.loss, loss);
    if (failed && tid == 0) {
        atomicAdd(a.err, 1u);
        mbar_wait(mbar, phase ^ 1u, kWaitPolls);   // the commit that did not arrive, once more
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem, kTrainTmemCols);
    }
}

// ---------------------------------------------------------------- parameters
__device__ __forceinline__ float hash01(uint32_t seed, uint32_t i)
{
    return (float)(ff_wang_hash(ff_wang_hash(seed) ^ (i * 0x9E3779B9u + 0x7F4A7C15u)) >> 8) * (1.f / 16777216.f);
}

__global__ void k_init_grid(float2* __restrict__ table, __half2* __restrict__ table_h, uint32_t n, uint32_t seed)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 v = make_float2((hash01(seed, 2 * i) * 2.f - 1.f) * 1e-4f, (hash01(seed, 2 * i + 1) * 2.f - 1.f) * 1e-4f);
    table[i] = v;
    table_h[i] = __floats2half2_rn(v.x, v.y);
}

// Xavier-uniform weights; rows 3..63 of the output layer are zero.
__global__ void k_init_mlp(float* __restrict__ w, uint32_t seed)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const uint32_t l = i / (kWidth * kWidth), row = (i / kWidth) % kWidth;
    const float fan_out = l == kLayers - 1 ? (float)kOutputs : (float)kWidth;
    const float lim = sqrtf(6.f / ((float)kWidth + fan_out));
    w[i] = (l == kLayers - 1 && row >= (uint32_t)kOutputs) ? 0.f : (hash01(seed ^ 0xA5A5A5A5u, i) * 2.f - 1.f) * lim;
}

__device__ __forceinline__ void put_image(uint8_t* img, uint32_t i, float w)
{
    const uint32_t l = i / (kWidth * kWidth), row = (i / kWidth) % kWidth, col = i % kWidth;
    *reinterpret_cast<__nv_bfloat16*>(img + l * kWBytes + sw128_offset(row, col)) = __float2bfloat16_rn(w);
}

__global__ void k_pack_mlp(const float* __restrict__ w, uint8_t* __restrict__ img)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kParams) put_image(img, i, w[i]);
}

struct AdamHP {
    float lr, b1, b2, eps, c1, c2;      // c1 = 1 - b1^t, c2 = 1 - b2^t
};

__global__ void k_adam_mlp(float* __restrict__ w, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                           uint8_t* __restrict__ img, AdamHP hp)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float gi = g[i];
    g[i] = 0.f;
    const uint32_t l = i / (kWidth * kWidth), row = (i / kWidth) % kWidth;
    if (l == kLayers - 1 && row >= (uint32_t)kOutputs) return;
    const float mi = hp.b1 * m[i] + (1.f - hp.b1) * gi;
    const float vi = hp.b2 * v[i] + (1.f - hp.b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - hp.lr * (mi / hp.c1) / (sqrtf(vi / hp.c2) + hp.eps);
    w[i] = wi;
    put_image(img, i, wi);
}

// Sparse Adam over the grid: entries no record touched keep their state.
__global__ void k_adam_grid(float2* __restrict__ table, __half2* __restrict__ table_h, float2* __restrict__ g,
                            float2* __restrict__ m, float2* __restrict__ v, uint32_t n, AdamHP hp)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 gi = g[i];
    if (gi.x == 0.f && gi.y == 0.f) return;
    g[i] = make_float2(0.f, 0.f);
    float2 mi = m[i], vi = v[i], p = table[i];
    mi.x = hp.b1 * mi.x + (1.f - hp.b1) * gi.x;
    mi.y = hp.b1 * mi.y + (1.f - hp.b1) * gi.y;
    vi.x = hp.b2 * vi.x + (1.f - hp.b2) * gi.x * gi.x;
    vi.y = hp.b2 * vi.y + (1.f - hp.b2) * gi.y * gi.y;
    p.x -= hp.lr * (mi.x / hp.c1) / (sqrtf(vi.x / hp.c2) + hp.eps);
    p.y -= hp.lr * (mi.y / hp.c1) / (sqrtf(vi.y / hp.c2) + hp.eps);
    m[i] = mi;
    v[i] = vi;
    table[i] = p;
    table_h[i] = __floats2half2_rn(p.x, p.y);
}

__global__ void k_half_of(const float2* __restrict__ table, __half2* __restrict__ table_h, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) table_h[i] = __floats2half2_rn(table[i].x, table[i].y);
}

unsigned grid_for(size_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

}  // namespace

// ---------------------------------------------------------------- host side
void ff_cache_setup_grid(ff_cache* c)
{
    Grid& g = c->grid;
    g.table_h = c->table_h.as<__half2>();
    g.grad = c->grid_grad.as<float2>();
    g.log2_T = c->prm.log2_table_size;
    const float3 lo = c->lo, hi = c->hi;
    const float3 ext = make_float3(fmaxf(hi.x - lo.x, 1e-6f), fmaxf(hi.y - lo.y, 1e-6f), fmaxf(hi.z - lo.z, 1e-6f));
    g.lo = lo;
    g.inv_ext = make_float3(1.f / ext.x, 1.f / ext.y, 1.f / ext.z);
    const double b = std::exp((std::log((double)c->prm.max_resolution) - std::log((double)c->prm.base_resolution)) /
                              (kLevels - 1));
    const uint64_t T = 1ull << g.log2_T;
    for (int l = 0; l < kLevels; ++l) {
        const uint32_t cells = (uint32_t)std::floor((double)c->prm.base_resolution * std::pow(b, l) + 1e-9);
        g.scale[l] = (float)cells;
        const uint64_t side = (uint64_t)cells + 1;
        g.dense_side[l] = side * side * side <= T ? (uint32_t)side : 0u;
    }
}

void ff_cache_init_params(ff_cache* c)
{
    cudaStream_t st = c->ctx->stream;
    const uint32_t n = kLevels << c->prm.log2_table_size;
    k_init_grid<<<grid_for(n, 256), 256, 0, st>>>(c->table.as<float2>(), c->table_h.as<__half2>(), n, c->prm.seed);
    k_init_mlp<<<grid_for(kParams, 256), 256, 0, st>>>(c->mlp.as<float>(), c->prm.seed);
    k_pack_mlp<<<grid_for(kParams, 256), 256, 0, st>>>(c->mlp.as<float>(), c->mlp_img.as<uint8_t>());
    FF_CUDA_CHECK(cudaMemsetAsync(c->grid_grad.ptr, 0, sizeof(float2) * n, st));
    FF_CUDA_CHECK(cudaMemsetAsync(c->grid_m.ptr, 0, sizeof(float2) * n, st));
    FF_CUDA_CHECK(cudaMemsetAsync(c->grid_v.ptr, 0, sizeof(float2) * n, st));
    FF_CUDA_CHECK(cudaMemsetAsync(c->mlp_grad.ptr, 0, sizeof(float) * kParams, st));
    FF_CUDA_CHECK(cudaMemsetAsync(c->mlp_m.ptr, 0, sizeof(float) * kParams, st));
    FF_CUDA_CHECK(cudaMemsetAsync(c->mlp_v.ptr, 0, sizeof(float) * kParams, st));
    FF_CUDA_CHECK(cudaGetLastError());
    c->step = 0;
}

// The dynamic shared memory above 48 KB is an attribute of the kernel on each
// device: set once per (kernel, device).
static void allow_smem(ff_cache* c, const void* fn, uint32_t bytes, int which)
{
    static std::atomic<uint64_t> done[2];
    const uint64_t bit = 1ull << (c->ctx->device & 63);
    if (done[which].load() & bit) return;
    FF_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done[which].fetch_or(bit);
}

static CacheArgs make_args(ff_cache* c, const Record* recs, uint32_t n, const uint32_t* n_dev)
{
    CacheArgs a{};
    a.grid = c->grid;
    a.w_img = c->mlp_img.as<uint4>();
    a.recs = recs;
    a.n_dev = n_dev;
    a.n = n;
    a.grad_w = c->mlp_grad.as<float>();
    a.loss = c->loss.as<float>();
    a.err = c->err.as<unsigned int>();
    a.wait_polls = c->wait_polls == FF_DEBUG_WAIT_DEFAULT ? kWaitPolls : c->wait_polls;
    return a;
}

void ff_cache_launch_infer(ff_cache* c, const void* recs, uint32_t n_max, const uint32_t* n_dev, float* out_rgb,
                           float4* frame)
{
    allow_smem(c, reinterpret_cast<const void*>(k_cache_infer), kInferSmem, 0);
    if (n_max == 0) return;
    CacheArgs a = make_args(c, static_cast<const Record*>(recs), n_max, n_dev);
    a.out_rgb = out_rgb;
    a.frame = frame;
    const uint32_t tiles = (n_max + kTile - 1) / kTile;
    const uint32_t grid = std::min<uint32_t>((tiles + kGroups - 1) / kGroups, (uint32_t)c->ctx->num_sms * 2u);
    k_cache_infer<<<grid, kInferThreads, kInferSmem, c->ctx->stream>>>(a);
    FF_CUDA_CHECK(cudaGetLastError());
}

// Gradients of the batch (added to the accumulators) and, unless
// gradients_only, one Adam step of the MLP and the grid.  With n_dev the
// batch is records [offset, offset + n_max) of a list whose length is on the
// device, and the loss is normalised by the records actually present.
static void launch_train(ff_cache* c, const Record* recs, uint32_t offset, uint32_t n_max, const uint32_t* n_dev,
                         uint32_t n_norm, bool gradients_only, cudaStream_t st)
{
    allow_smem(c, reinterpret_cast<const void*>(k_cache_train), kTrainSmem, 1);
    if (n_max == 0) return;
    CacheArgs a = make_args(c, recs + offset, n_max, n_dev);
    a.offset = offset;
    a.inv_n = 1.f / (float)std::max<uint32_t>(n_norm, 1u);
    const uint32_t tiles = (n_max + kTile - 1) / kTile;
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)c->ctx->num_sms);
    k_cache_train<<<grid, kThreads, kTrainSmem, st>>>(a);
    FF_CUDA_CHECK(cudaGetLastError());
    if (gradients_only) return;
    c->step += 1;
    AdamHP hp;
    hp.lr = c->prm.lr;
    hp.b1 = c->prm.beta1;
    hp.b2 = c->prm.beta2;
    hp.eps = c->prm.eps;
    hp.c1 = 1.f - (float)std::pow((double)hp.b1, (double)c->step);
    hp.c2 = 1.f - (float)std::pow((double)hp.b2, (double)c->step);
    k_adam_mlp<<<grid_for(kParams, 256), 256, 0, st>>>(c->mlp.as<float>(), c->mlp_grad.as<float>(), c->mlp_m.as<float>(),
                                                      c->mlp_v.as<float>(), c->mlp_img.as<uint8_t>(), hp);
    const uint32_t ng = kLevels << c->prm.log2_table_size;
    k_adam_grid<<<grid_for(ng, 256), 256, 0, st>>>(c->table.as<float2>(), c->table_h.as<__half2>(),
                                                  c->grid_grad.as<float2>(), c->grid_m.as<float2>(),
                                                  c->grid_v.as<float2>(), ng, hp);
    FF_CUDA_CHECK(cudaGetLastError());
}

void ff_cache_launch_train(ff_cache* c, const void* recs, uint32_t n, bool gradients_only)
{
    launch_train(c, static_cast<const Record*>(recs), 0, n, nullptr, n, gradients_only, c->ctx->stream);
}

void ff_cache_launch_train_slice(ff_cache* c, const void* recs, uint32_t offset, uint32_t n_max, const uint32_t* n_dev,
                                 cudaStream_t st)
{
    launch_train(c, static_cast<const Record*>(recs), offset, n_max, n_dev, n_max, false, st);
}

void ff_cache_refresh_copies(ff_cache* c)
{
    cudaStream_t st = c->ctx->stream;
    const uint32_t n = kLevels << c->prm.log2_table_size;
    k_half_of<<<grid_for(n, 256), 256, 0, st>>>(c->table.as<float2>(), c->table_h.as<__half2>(), n);
    k_pack_mlp<<<grid_for(kParams, 256), 256, 0, st>>>(c->mlp.as<float>(), c->mlp_img.as<uint8_t>());
    FF_CUDA_CHECK(cudaGetLastError());
}

uint32_t ff_cache_num_params() { return kParams; }
