// ff_cache.cuh — inputs of the learned radiance cache: the multiresolution
// hash-grid encoding of the position (16 levels x 2 features, 2^19 entries
// per level), degree-4 real spherical harmonics (16 coefficients) of the
// outgoing direction, the shading normal and the roughness, assembled into
// the 64 inputs of the MLP:
//   0..31  hash features, level l at 2l, 2l+1
//   32..47 SH(wo)
//   48..50 normal, 51 roughness, 52 constant 1 (the first layer's bias)
//   53..63 zero
#pragma once

#include <cuda_fp16.h>

#include "ff_common.cuh"

namespace ffc {

constexpr int kLevels = 16;
constexpr int kInputs = 64;
constexpr int kWidth = 64;
constexpr int kLayers = 5;          // 4 hidden layers of 64 (W0..W3) and the output layer W4
constexpr int kOutputs = 3;
constexpr int kTile = 128;          // records per tensor-core tile (M)

struct Grid {
    const __half2* table_h;         // [kLevels << log2_T] features used by the MLP
    float2* grad;                   // [kLevels << log2_T] gradient accumulator (training)
    uint32_t log2_T;
    float3 lo, inv_ext;             // position normalisation (scene box)
    float scale[kLevels];           // cells per unit cube side at each level
    uint32_t dense_side[kLevels];   // side+1 of a densely indexed level, 0 for hashed levels
};

// One record: a vertex (position, roughness, outgoing direction, normal)
// and a value (training: target radiance; render queries: path throughput).
struct alignas(16) Record {
    float px, py, pz, rough;
    float wx, wy, wz, v0;
    float nx, ny, nz, v1;
    uint32_t pixel;
    float v2, pad0, pad1;
};
static_assert(sizeof(Record) == 64, "record layout");

__device__ __forceinline__ Record make_record(float3 pos, float rough, float3 wo, float3 n, float3 v, uint32_t pixel)
{
    Record r;
    r.px = pos.x;
    r.py = pos.y;
    r.pz = pos.z;
    r.rough = rough;
    r.wx = wo.x;
    r.wy = wo.y;
    r.wz = wo.z;
    r.v0 = v.x;
    r.nx = n.x;
    r.ny = n.y;
    r.nz = n.z;
    r.v1 = v.y;
    r.pixel = pixel;
    r.v2 = v.z;
    r.pad0 = r.pad1 = 0.f;
    return r;
}

__device__ __forceinline__ float3 normalised_pos(const Grid& g, float px, float py, float pz)
{
    float3 p = make_float3((px - g.lo.x) * g.inv_ext.x, (py - g.lo.y) * g.inv_ext.y, (pz - g.lo.z) * g.inv_ext.z);
    p.x = fminf(fmaxf(p.x, 0.f), 1.f);
    p.y = fminf(fmaxf(p.y, 0.f), 1.f);
    p.z = fminf(fmaxf(p.z, 0.f), 1.f);
    return p;
}

// The 8 corners of the level-l cell holding p: table indices and trilinear
// weights (corner bit 0 = +x, bit 1 = +y, bit 2 = +z).
struct Corners {
    uint32_t idx[8];
    float w[8];
};

__device__ __forceinline__ void level_corners(const Grid& g, int l, float3 p, Corners& c)
{
    const float s = g.scale[l];
    const float fx = p.x * s, fy = p.y * s, fz = p.z * s;
    const int cells = (int)s;
    int ix = min((int)floorf(fx), cells - 1), iy = min((int)floorf(fy), cells - 1), iz = min((int)floorf(fz), cells - 1);
    ix = max(ix, 0);
    iy = max(iy, 0);
    iz = max(iz, 0);
    const float tx = fminf(fmaxf(fx - (float)ix, 0.f), 1.f);
    const float ty = fminf(fmaxf(fy - (float)iy, 0.f), 1.f);
    const float tz = fminf(fmaxf(fz - (float)iz, 0.f), 1.f);
    const uint32_t side = g.dense_side[l];
    const uint32_t mask = (1u << g.log2_T) - 1u;
    const uint32_t base = (uint32_t)l << g.log2_T;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t x = (uint32_t)ix + (k & 1), y = (uint32_t)iy + ((k >> 1) & 1), z = (uint32_t)iz + (k >> 2);
        uint32_t i;
        if (side) i = x + side * (y + side * z);
        else i = (x * 1u) ^ (y * 2654435761u) ^ (z * 805459861u);
        c.idx[k] = base + (i & mask);
        c.w[k] = ((k & 1) ? tx : 1.f - tx) * (((k >> 1) & 1) ? ty : 1.f - ty) * ((k >> 2) ? tz : 1.f - tz);
    }
}

// Entry j (0..3) of four packed half2 entries.
__device__ __forceinline__ uint32_t pick4(uint4 q, uint32_t j)
{
    return j == 0u ? q.x : (j == 1u ? q.y : (j == 2u ? q.z : q.w));
}
__device__ __forceinline__ float2 half2_bits(uint32_t u)
{
    __half2 h;
    *reinterpret_cast<uint32_t*>(&h) = u;
    return __half22float2(h);
}

// Trilinear feature of level l at p.  Corners k (x) and k + 1 (x + 1) share
// y and z, so their entries usually sit in one aligned group of four: on a
// dense level they are neighbours, and on a hashed level x enters the hash
// by XOR, so the two indices differ in the bits of x ^ (x + 1), which stay
// below 4 three times in four.  The group is one 16-byte load (one sector
// per lane instead of two); an entry outside it is read alone.  The sum runs
// over the corners in the same order, so the feature is unchanged.
__device__ __forceinline__ float2 level_feature(const Grid& g, int l, float3 p)
{
    Corners c;
    level_corners(g, l, p, c);
    float2 f = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 8; k += 2) {
        const uint32_t i0 = c.idx[k], i1 = c.idx[k + 1];
        const uint4 q = *reinterpret_cast<const uint4*>(g.table_h + (i0 & ~3u));
        const uint32_t b1 = (i0 ^ i1) < 4u ? pick4(q, i1 & 3u) : *reinterpret_cast<const uint32_t*>(g.table_h + i1);
        const float2 e0 = half2_bits(pick4(q, i0 & 3u)), e1 = half2_bits(b1);
        f.x += c.w[k] * e0.x;
        f.y += c.w[k] * e0.y;
        f.x += c.w[k + 1] * e1.x;
        f.y += c.w[k + 1] * e1.y;
    }
    return f;
}

// Real spherical harmonics of degree 0..3 (16 functions) of the unit
// direction (x, y, z), in the order (l, m) = (0,0), (1,-1), (1,0), (1,1),
// (2,-2) .. (2,2), (3,-3) .. (3,3); normalisation constants from
// sqrt((2l+1)/(4 pi) * (l-|m|)!/(l+|m|)!), with the Condon-Shortley phase.
__device__ __forceinline__ void sh16(float x, float y, float z, float* o)
{
    const float c00 = (float)(0.5 / 1.7724538509055160273);                 // 1/(2 sqrt(pi))
    const float c1 = (float)(0.48860251190291992159);                       // sqrt(3/(4 pi))
    const float c2a = (float)(1.0925484305920790705);                       // sqrt(15/pi)/2
    const float c2b = (float)(0.31539156525252000603);                      // sqrt(5/pi)/4
    const float c2c = (float)(0.54627421529603953527);                      // sqrt(15/pi)/4
    const float c3a = (float)(0.59004358992664351035);                      // sqrt(35/(2 pi))/4
    const float c3b = (float)(2.8906114426405540554);                       // sqrt(105/pi)/2
    const float c3c = (float)(0.45704579946446573616);                      // sqrt(21/(2 pi))/4
    const float c3d = (float)(0.37317633259011539141);                      // sqrt(7/pi)/4
    const float c3e = (float)(1.4453057213202770277);                       // sqrt(105/pi)/4
    const float xx = x * x, yy = y * y, zz = z * z;
    o[0] = c00;
    o[1] = -c1 * y;
    o[2] = c1 * z;
    o[3] = -c1 * x;
    o[4] = c2a * x * y;
    o[5] = -c2a * y * z;
    o[6] = c2b * (3.f * zz - 1.f);
    o[7] = -c2a * x * z;
    o[8] = c2c * (xx - yy);
    o[9] = -c3a * y * (3.f * xx - yy);
    o[10] = c3b * x * y * z;
    o[11] = -c3c * y * (5.f * zz - 1.f);
    o[12] = c3d * z * (5.f * zz - 3.f);
    o[13] = -c3c * x * (5.f * zz - 1.f);
    o[14] = c3e * z * (xx - yy);
    o[15] = -c3a * x * (xx - 3.f * yy);
}

}  // namespace ffc
