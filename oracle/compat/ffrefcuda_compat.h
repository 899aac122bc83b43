/*
 * ffrefcuda_compat.h — forced-include shim that lets the reference's device
 * traversal (JakeKurtz/Firefly, CUDA-RayTracer/dTriangle.cu and dRay.cu)
 * compile unmodified with nvcc for sm_100a.  TEST INFRASTRUCTURE ONLY: it
 * builds oracle/_ref/libffrefcuda.so, the reference's own GPU code, timed as
 * the "reference CUDA" baseline beside the product's trace kernel.
 *
 * What it changes, and why:
 *  - glibc's M_* macros collide with the constants dMath.cuh defines
 *    (dMath.cuh:83-128): include libm first, then undefine them.
 *  - __any() is the pre-Volta warp vote the reference calls in intersect()
 *    (dTriangle.cu:167); sm_70+ only has __any_sync.  Over the lanes active at
 *    that point (those at a leaf), __any_sync(__activemask(), x) is what
 *    __any(x) meant.
 *  - glm is absent: the stub under oracle/compat/glm serves dMath.cuh's include.
 */
#ifndef FFREFCUDA_COMPAT_H
#define FFREFCUDA_COMPAT_H

#include <math.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <cuda_runtime.h>

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

#define __any(x) __any_sync(__activemask(), (x))

#endif
