// ff_common.cuh — shared device definitions of the B200 wavefront path tracer:
// vector helpers, the seeded sampler, and the layouts of the 8-wide BVH and the
// triangle records in HBM.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "firefly_b200.h"

#define FF_HD __host__ __device__ __forceinline__
#define FF_D __device__ __forceinline__

// K_EPSILON and K_HUGE of the reference (CUDA-RayTracer/dMath.cuh:78,80).
#define FF_K_EPSILON 1e-6f
#define FF_K_HUGE 1e32f
// The reference's float pi constants (dMath.cuh:103-122 declare them float).
#define FF_PI 3.14159265358979323846f
#define FF_2PI 6.28318530717958647692f
#define FF_PI_2 1.57079632679489661923f
#define FF_PI_4 0.785398163397448309615f
#define FF_1_PI 0.318309886183790671537f
#define FF_1_2PI 0.159154943091895335768f
#define FF_1_4PI 0.0795774715459476678844f

// ------------------------------------------------------------------ float3
FF_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
FF_HD float3 f3(float s) { return make_float3(s, s, s); }
FF_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
FF_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
FF_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
FF_HD float3 operator-(float s, float3 a) { return make_float3(s - a.x, s - a.y, s - a.z); }
FF_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
FF_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
FF_HD float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
FF_HD float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
FF_HD float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
FF_HD float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
FF_HD float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
FF_HD float3& operator*=(float3& a, float s) { a = a * s; return a; }
FF_HD bool operator==(float3 a, float3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
FF_HD bool operator!=(float3 a, float3 b) { return !(a == b); }
FF_HD float3 fmin3(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
FF_HD float3 fmax3(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
FF_HD float comp(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// Round-to-nearest helpers that the compiler may not contract into FMAs.  The
// reference's host build evaluates every vector expression with one rounding
// per operation (x86-64 SSE), so these reproduce it bit for bit.
FF_D float rn_dot(float3 a, float3 b)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
FF_D float3 rn_cross(float3 a, float3 b)
{
    return make_float3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
                       __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
                       __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
FF_D float3 rn_sub(float3 a, float3 b)
{
    return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}

// ----------------------------------------------------------------- sampler
// wang_hash of the reference (CUDA-RayTracer/dRandom.cu:10-18).
FF_HD uint32_t ff_wang_hash(uint32_t s)
{
    s = (s ^ 61u) ^ (s >> 16);
    s *= 9u;
    s = s ^ (s >> 4);
    s *= 0x27d4eb2du;
    s = s ^ (s >> 15);
    return s;
}
// The reference's random() is wang_hash of a clock()-based seed scaled by
// 2^-32 and returned as float (dRandom.cu:20-27).  The seeded replacement
// keeps the hash and the conversion and indexes draws by (path key, sample
// dimension) instead of the clock, so every draw is reproducible:
// u = float(wang_hash(key ^ wang_hash(dim)) * 2^-32).  The conversion rounds
// to nearest and can return 1.0f, as the reference's can.
FF_D float ff_rand(uint32_t key, uint32_t dim)
{
    uint32_t h = ff_wang_hash(key ^ ff_wang_hash(dim));
    return __uint2float_rn(h) * 2.3283064365386963e-10f;  // exact power-of-two scale
}
FF_HD uint32_t ff_path_key(uint32_t seed, uint32_t pixel, uint32_t sample)
{
    return ff_wang_hash(ff_wang_hash(ff_wang_hash(seed) ^ pixel) + sample);
}

// ------------------------------------------------------------- BVH layout
// 8-wide BVH node with 8-bit quantised child boxes (80 bytes, five 16-byte
// loads).  Child box of slot s on axis a spans
//   [p_a + qlo_a[s] * 2^e_a,  p_a + qhi_a[s] * 2^e_a]
// and contains the exact child bounds padded by at least one grid step.
// Internal children of a node are stored contiguously from child_base in slot
// order; child of slot s is child_base + popc(imask & ((1<<s)-1)).  Leaf
// children own up to 3 consecutive triangle records starting at
// tri_base + (meta[s] & 31); meta[s] >> 5 is a unary count (1, 3, 7).  An
// unused slot has meta 0.
struct __align__(16) FFNode8 {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlox[8];
    uint8_t qloy[8];
    uint8_t qloz[8];
    uint8_t qhix[8];
    uint8_t qhiy[8];
    uint8_t qhiz[8];
};
static_assert(sizeof(FFNode8) == 80, "FFNode8 must be 80 bytes");

// Triangle record for traversal (48 bytes, three 16-byte loads):
//   a = (v0.xyz, original index as int bits), b = (v1 - v0, 0), c = (v2 - v0, 0).
// e1 and e2 are rounded once, exactly as the reference rounds them at every
// test (dTriangle.cu:35-36), so precomputing them changes no result.
struct __align__(16) FFTri {
    float4 a, b, c;
};

// Box-test widening: a child box is entered when
//   max(tnear - |tnear|*W, tmin) <= min(tfar + |tfar|*W, tbest + |tbest|*W).
// W covers the float rounding of the slab test and the reference test's own
// acceptance slack, so pruning never drops a triangle that the reference
// routine reports as the closest (or any) hit.
#define FF_BOX_WIDEN 2.44140625e-4f  // 2^-12

// Bit 31 of a triangle index marks a back-face hit of a two-sided ray
// (FFRayState::prim, and the material word of a path vertex).
constexpr uint32_t kBackFace = 0x80000000u;

struct FFBvhView {
    const FFNode8* nodes;
    const FFTri* tris;
    uint32_t num_nodes;
    uint32_t num_tris;
};
