/*
 * ffref_compat.h — forced-include shim that lets the reference's device
 * routines (JakeKurtz/Firefly, CUDA-RayTracer/*.cu) compile as host C++ with
 * g++.  TEST INFRASTRUCTURE ONLY: it builds oracle/_ref/libffref.so, the
 * reference's own code, used to pin the oracle and as the timed CPU baseline.
 *
 * What it changes, and why:
 *  - glibc's M_* macros and random() collide with names the reference
 *    defines (dMath.cuh:83-128, dRandom.cu:20): include libm first, then
 *    undefine the macros and rename random.
 *  - dMath.cuh defines host fminf/fmaxf (under !__CUDACC__, :40-48) with the
 *    same signature as libm's: rename them, so the reference's own host
 *    versions are the ones used.
 *  - threadIdx/blockIdx/blockDim, clock(), __any(), tex2DLod and
 *    surf2Dread are device built-ins: provide host stand-ins.  clock()
 *    returns values from a sequence the harness sets, so random() draws are
 *    controlled (random() hashes (thread index, clock()), dRandom.cu:20-27).
 *  - glm, curand and the Windows allocator header are absent: small stubs
 *    under oracle/compat/.
 */
#ifndef FFREF_COMPAT_H
#define FFREF_COMPAT_H

#include <math.h>
#include <cmath>
#include <cstdlib>
#include <stdlib.h>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <cstdint>
#include <climits>
#include <limits>
#include <algorithm>
#include <vector>
#include <string>
#include <list>
#include <cuda_runtime.h>
#include <vector_functions.h>

#undef M_E
#undef M_LOG2E
#undef M_LOG10E
#undef M_LN2
#undef M_LN10
#undef M_PI
#undef M_PI_2
#undef M_PI_4
#undef M_1_PI
#undef M_2_PI
#undef M_2_SQRTPI
#undef M_SQRT2
#undef M_SQRT1_2

#define random ffref_random
#define fminf ffref_fminf
#define fmaxf ffref_fmaxf

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;

/* clock(): values from a harness-controlled sequence. */
long ffref_clock(void);
#define clock() ffref_clock()

#define __any(x) (x)

/* Host texture / surface emulation (texture objects are registry ids). */
void ffref_tex_fetch(unsigned long long obj, float u, float v, float out[4]);
void ffref_surf_read_float(unsigned long long obj, int x_bytes, int y, float* out);

template <class T>
T tex2DLod(unsigned long long obj, float u, float v, float lod);
template <>
inline float4 tex2DLod<float4>(unsigned long long obj, float u, float v, float lod)
{
    (void)lod;
    float o[4];
    ffref_tex_fetch(obj, u, v, o);
    return make_float4(o[0], o[1], o[2], o[3]);
}
inline void surf2Dread(float* out, unsigned long long obj, int x_bytes, int y)
{
    ffref_surf_read_float(obj, x_bytes, y, out);
}

#endif
