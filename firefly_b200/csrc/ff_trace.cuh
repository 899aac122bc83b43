// ff_trace.cuh — ray traversal of the 8-wide quantised BVH and the
// reference-exact ray/triangle tests.  Used by the standalone trace kernel
// (ff_trace.cu) and by the wavefront stages.
#pragma once

#include "ff_common.cuh"

// Per-ray traversal state kept in registers.
//
// Two-sided closest hits (rays inside a refracting object, and ff_trace with
// FF_TRACE_TWO_SIDED) ride on the sign bit of tmin in the traversal kernels
// instantiated with TWO = true: a ray whose tmin has its sign bit set (-0.0
// for tmin 0) also accepts back faces, and such a ray's interval starts at
// |tmin|.  A back-face hit keeps bit 31 of prim set.  Kernels with TWO =
// false never look at the sign and cull back faces as the reference does.
struct FFRayState {
    float3 o, d, inv;
    float tmin, tmax;   // closest-hit: tmax is the current best t (starts at min(tmax, K_HUGE))
    float u, v;
    uint32_t prim;      // original triangle index, 0xffffffff = none; bit 31: back face (TWO kernels)
    uint32_t oct_inv;   // 7 ^ octant of d (bit a set = d_a < 0)
};

// A closest hit as the C ABI reports it: prim = the original index for a
// front face, -2 - index for a back face of a two-sided ray, -1 for none.
FF_D ff_hit ff_hit_of(const FFRayState& r)
{
    int32_t prim = -1;
    if (r.prim != 0xffffffffu) {
        const int32_t id = (int32_t)(r.prim & ~kBackFace);
        prim = (r.prim & kBackFace) ? -2 - id : id;
    }
    return ff_hit{r.tmax, r.u, r.v, prim};
}

FF_D float safe_inv(float x)
{
    const float tiny = 1e-20f;
    return 1.0f / (fabsf(x) > tiny ? x : copysignf(tiny, x));
}

FF_D void ff_ray_setup(FFRayState& r, float3 o, float3 d, float tmin, float tmax, bool any)
{
    r.o = o;
    r.d = d;
    r.inv = make_float3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    r.tmin = tmin;
    r.tmax = any ? tmax : fminf(tmax, FF_K_HUGE);
    r.u = r.v = 0.f;
    r.prim = 0xffffffffu;
    r.oct_inv = (d.x < 0.f ? 0u : 1u) | (d.y < 0.f ? 0u : 2u) | (d.z < 0.f ? 0u : 4u);
}

FF_D uint32_t byte_of(uint32_t lo4, uint32_t hi4, int s)
{
    return ((s < 4 ? lo4 : hi4) >> (8 * (s & 3))) & 0xffu;
}

// Byte s of (lo4, hi4) as a float, without an integer-to-float conversion:
// one byte permute builds the float 2^23 + byte (exponent byte 0x4B, the byte
// in the low mantissa bits), one subtraction removes 2^23.  Exact for 0..255.
FF_D float byte_as_float(uint32_t lo4, uint32_t hi4, int s)
{
    const uint32_t bits = __byte_perm(s < 4 ? lo4 : hi4, 0x4B000000u, 0x7440u | (uint32_t)(s & 3));
    return __uint_as_float(bits) - 8388608.0f;
}

// Byte s of (lo4, hi4) as the float 2^23 + byte (one byte permute); the
// node test subtracts 2^23 from two such values with one packed add.
FF_D float byte_plus_2p23(uint32_t lo4, uint32_t hi4, int s)
{
    return __uint_as_float(__byte_perm(s < 4 ? lo4 : hi4, 0x4B000000u, 0x7440u | (uint32_t)(s & 3)));
}

// Three-input min / max of sm_100 (one instruction instead of two; exact,
// and NaN-ignoring like fminf / fmaxf).
FF_D float fmin3f(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
FF_D float fmax3f(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Intersect the ray with the 8 child boxes of node idx.  Returns the new node
// group (x = child_base, y = hit bits 24..31 in traversal order | imask) and
// the triangle group (x = tri_base, y = 24-bit mask of triangles to test).
FF_D void ff_intersect_node(const FFNode8* __restrict__ nodes, uint32_t idx, const FFRayState& r,
                            uint2& node_group, uint2& tri_group)
{
    const uint4* p = reinterpret_cast<const uint4*>(nodes + idx);
    const uint4 n0 = __ldg(p + 0);
    const uint4 n1 = __ldg(p + 1);
    const uint4 n2 = __ldg(p + 2);
    const uint4 n3 = __ldg(p + 3);
    const uint4 n4 = __ldg(p + 4);
    const float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    const uint32_t ex = n0.w & 0xffu, ey = (n0.w >> 8) & 0xffu, ez = (n0.w >> 16) & 0xffu;
    const uint32_t imask = n0.w >> 24;
    const float sx = __uint_as_float(ex << 23), sy = __uint_as_float(ey << 23), sz = __uint_as_float(ez << 23);
    const float ax = sx * r.inv.x, ay = sy * r.inv.y, az = sz * r.inv.z;
    const float bx = (px - r.o.x) * r.inv.x, by = (py - r.o.y) * r.inv.y, bz = (pz - r.o.z) * r.inv.z;
    // near/far plane words per axis, chosen by the sign of the direction
    const uint32_t nx0 = r.inv.x >= 0.f ? n2.x : n3.z, nx1 = r.inv.x >= 0.f ? n2.y : n3.w;
    const uint32_t fx0 = r.inv.x >= 0.f ? n3.z : n2.x, fx1 = r.inv.x >= 0.f ? n3.w : n2.y;
    const uint32_t ny0 = r.inv.y >= 0.f ? n2.z : n4.x, ny1 = r.inv.y >= 0.f ? n2.w : n4.y;
    const uint32_t fy0 = r.inv.y >= 0.f ? n4.x : n2.z, fy1 = r.inv.y >= 0.f ? n4.y : n2.w;
    const uint32_t nz0 = r.inv.z >= 0.f ? n3.x : n4.z, nz1 = r.inv.z >= 0.f ? n3.y : n4.w;
    const uint32_t fz0 = r.inv.z >= 0.f ? n4.z : n3.x, fz1 = r.inv.z >= 0.f ? n4.w : n3.y;
    // the widening as explicit fused multiply-adds: the same result in every
    // translation unit, whatever its contraction setting (-fmad)
    const float tb = __fmaf_rn(fabsf(r.tmax), FF_BOX_WIDEN, r.tmax);
    // x and y in packed FP32: one add removes 2^23 from two plane bytes and
    // one fma gives two slab distances (the same IEEE operations per lane as
    // fmaf, so the same values); z in scalar fmaf
    const float2 axy = make_float2(ax, ay), bxy = make_float2(bx, by);
    const float2 m23 = make_float2(-8388608.0f, -8388608.0f);
    uint32_t hits = 0, tmask = 0;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const float2 qn = __fadd2_rn(make_float2(byte_plus_2p23(nx0, nx1, s), byte_plus_2p23(ny0, ny1, s)), m23);
        const float2 qf = __fadd2_rn(make_float2(byte_plus_2p23(fx0, fx1, s), byte_plus_2p23(fy0, fy1, s)), m23);
        const float2 qz = __fadd2_rn(make_float2(byte_plus_2p23(nz0, nz1, s), byte_plus_2p23(fz0, fz1, s)), m23);
        const float2 tnxy = __ffma2_rn(qn, axy, bxy);
        const float2 tfxy = __ffma2_rn(qf, axy, bxy);
        const float tnz = fmaf(qz.x, az, bz);
        const float tfz = fmaf(qz.y, az, bz);
        float tn = fmax3f(tnxy.x, tnxy.y, tnz);
        float tf = fmin3f(tfxy.x, tfxy.y, tfz);
        tn = __fmaf_rn(-fabsf(tn), FF_BOX_WIDEN, tn);
        tf = __fmaf_rn(fabsf(tf), FF_BOX_WIDEN, tf);
        // an empty slot (meta 0, not internal) adds nothing even where its
        // degenerate box is hit, so no occupancy test is needed
        if (fmaxf(tn, r.tmin) <= fminf(tf, tb)) {
            const uint32_t meta = byte_of(n1.z, n1.w, s);
            if ((imask >> s) & 1u) hits |= 1u << (24 + (s ^ r.oct_inv));
            else tmask |= (meta >> 5) << (meta & 31u);
        }
    }
    node_group = make_uint2(n1.x, hits | imask);
    tri_group = make_uint2(n1.y, tmask);
}

// dTriangle::intersect with TEST_CULL (CUDA-RayTracer/dTriangle.cu:34-61),
// then dTriangle::hit's t < 0 rejection (:99) and intersect()'s strict
// t < tmin acceptance (:170), with ties to the lowest original index.  The
// edge tests compare float values, so they run in FP32 exactly as the
// reference's float-vs-double comparisons; the FP64 reciprocal and products
// run only for candidates that pass them.
//
// TWO: a ray with the sign bit of tmin set also takes back faces (no
// reference counterpart: the reference only culls).  A back face is a
// determinant at or below -K_EPSILON; the test then runs on the negated
// determinant and numerators (negation is exact), i.e. the mirror image of
// the front-face test, and the hit keeps kBackFace in prim.  Front faces go
// through exactly the arithmetic above.
template <bool TWO = false>
FF_D void ff_test_tri_closest(const FFTri* __restrict__ tris, uint32_t k, FFRayState& r)
{
    const float4 a = __ldg(&tris[k].a);
    const float4 b = __ldg(&tris[k].b);
    const float4 c = __ldg(&tris[k].c);
    const float3 v0 = make_float3(a.x, a.y, a.z);
    const float3 e1 = make_float3(b.x, b.y, b.z);
    const float3 e2 = make_float3(c.x, c.y, c.z);
    const float3 pvec = rn_cross(r.d, e2);
    float det = rn_dot(e1, pvec);
    float sg = 1.f;
    if (det < FF_K_EPSILON) {
        if (!TWO || !signbit(r.tmin) || !(det <= -FF_K_EPSILON)) return;
        sg = -1.f;
        det = -det;
    }
    const float3 tvec = rn_sub(r.o, v0);
    const float uf = TWO ? sg * rn_dot(tvec, pvec) : rn_dot(tvec, pvec);
    if (uf < 0.f || uf > det) return;
    const float3 qvec = rn_cross(tvec, e1);
    const float vf = TWO ? sg * rn_dot(r.d, qvec) : rn_dot(r.d, qvec);
    if (vf < 0.f || __fadd_rn(uf, vf) > det) return;
    const float tf = TWO ? sg * rn_dot(e2, qvec) : rn_dot(e2, qvec);
    const double inv_det = __drcp_rn((double)det);
    const float t = __double2float_rn(__dmul_rn((double)tf, inv_det));
    if (t < 0.f || !(t >= (TWO ? fabsf(r.tmin) : r.tmin))) return;
    const uint32_t id = (uint32_t)__float_as_int(a.w);
    const uint32_t best = TWO ? (r.prim & ~kBackFace) : r.prim;
    if (t < r.tmax || (t == r.tmax && r.prim != 0xffffffffu && id < best)) {
        r.tmax = t;
        r.prim = (TWO && sg < 0.f) ? (id | kBackFace) : id;
        r.u = __double2float_rn(__dmul_rn((double)uf, inv_det));
        r.v = __double2float_rn(__dmul_rn((double)vf, inv_det));
    }
}

// dTriangle::shadow_hit (CUDA-RayTracer/dTriangle.cu:110-138) and the
// t < tmin test of intersect_shadows (:233).  Returns true on an occluder.
// An FP32 pre-test rejects candidates that the FP64 test would certainly
// reject (sign of u, v and u + v > 1 with margin); the FP64 test decides the rest.
FF_D bool ff_test_tri_any(const FFTri* __restrict__ tris, uint32_t k, FFRayState& r)
{
    const float4 a = __ldg(&tris[k].a);
    const float4 b = __ldg(&tris[k].b);
    const float4 c = __ldg(&tris[k].c);
    const float3 v0 = make_float3(a.x, a.y, a.z);
    const float3 e1 = make_float3(b.x, b.y, b.z);
    const float3 e2 = make_float3(c.x, c.y, c.z);
    const float3 pvec = rn_cross(r.d, e2);
    const float det = rn_dot(e1, pvec);
    if (det > -FF_K_EPSILON && det < FF_K_EPSILON) return false;
    const float3 tvec = rn_sub(r.o, v0);
    const float uf = rn_dot(tvec, pvec);
    const bool neg = det < 0.f;
    if (uf != 0.f && ((uf < 0.f) != neg)) return false;  // u < 0
    const float3 qvec = rn_cross(tvec, e1);
    const float vf = rn_dot(r.d, qvec);
    if (vf != 0.f && ((vf < 0.f) != neg)) return false;  // v < 0
    if (fabsf(uf) + fabsf(vf) > fabsf(det) * 1.000001f) return false;  // u + v > 1
    const double inv_det = __drcp_rn((double)det);
    const double u = __dmul_rn((double)uf, inv_det);
    if (u < 0.0 || u > 1.0) return false;
    const double v = __dmul_rn((double)vf, inv_det);
    if (v < 0.0 || __dadd_rn(u, v) > 1.0) return false;
    const float tf = rn_dot(e2, qvec);
    const float t = __double2float_rn(__dmul_rn((double)tf, inv_det));
    if (t < 0.f) return false;
    if (t >= r.tmin && t < r.tmax) {
        r.prim = (uint32_t)__float_as_int(a.w);
        r.tmax = t;  // the traversal ends here; tmax now reports the occluder's t
        return true;
    }
    return false;
}

// Traversal stack: kShortStack entries per thread in shared memory (strided
// by the block size so a warp's pushes hit distinct banks), deeper entries in
// a local array.  Every push happens at most once per BVH level, so the depth
// needed is bounded by the BVH depth, which the host checks against
// kShortStack + kLocalStack at build time.
constexpr int kShortStack = 8;
constexpr int kLocalStack = 56;
constexpr int kMaxStack = kShortStack + kLocalStack;

struct FFStack {
    uint2* sm;     // this thread's column in shared memory
    int stride;    // block size
    int sp;
    bool overflow; // set instead of writing past the end (never expected: depth is checked at build)
    uint2 local[kLocalStack];
    FF_D void reset()
    {
        sp = 0;
        overflow = false;
    }
    FF_D void push(uint2 v)
    {
        if (sp >= kMaxStack) {
            overflow = true;
            return;
        }
        if (sp < kShortStack) sm[sp * stride] = v;
        else local[sp - kShortStack] = v;
        ++sp;
    }
    FF_D uint2 pop()
    {
        --sp;
        return sp < kShortStack ? sm[sp * stride] : local[sp - kShortStack];
    }
};

// Work counters for ff_traverse_step: FFNoCount compiles to nothing (the
// product kernels); FFCount tallies the node records fetched and the
// triangles tested (ff_trace_count).
struct FFNoCount {
    FF_D void node() {}
    FF_D void tri() {}
};
struct FFCount {
    unsigned long long nodes = 0, tris = 0;
    FF_D void node() { ++nodes; }
    FF_D void tri() { ++tris; }
};

// One traversal step: take the next child node of the current group, test
// its children, then test the triangles it exposed.  Returns true when the
// ray is finished.
template <bool ANY, class C, bool TWO = false>
FF_D bool ff_traverse_step(const FFBvhView& bvh, FFRayState& r, uint2& cur, FFStack& st, C& count)
{
    uint2 tri_group = make_uint2(0u, 0u);
    if (cur.y & 0xff000000u) {
        const uint32_t bit = 31u - __clz(cur.y & 0xff000000u);
        cur.y &= ~(1u << bit);
        const uint32_t slot = (bit - 24u) ^ r.oct_inv;
        const uint32_t child = cur.x + __popc(cur.y & 0xffu & ((1u << slot) - 1u));
        if (cur.y & 0xff000000u) st.push(cur);
        if (child >= bvh.num_nodes) {  // never taken on a validated BVH
            st.overflow = true;
            return true;
        }
        count.node();
        ff_intersect_node(bvh.nodes, child, r, cur, tri_group);
    }
    while (tri_group.y) {
        const uint32_t i = __ffs(tri_group.y) - 1;
        tri_group.y &= tri_group.y - 1;
        if (tri_group.x + i >= bvh.num_tris) {
            st.overflow = true;
            return true;
        }
        count.tri();
        if (ANY) {
            if (ff_test_tri_any(bvh.tris, tri_group.x + i, r)) return true;
        } else {
            ff_test_tri_closest<TWO>(bvh.tris, tri_group.x + i, r);
        }
    }
    if (!(cur.y & 0xff000000u)) {
        if (st.sp == 0) return true;
        cur = st.pop();
    }
    return st.overflow;
}
template <bool ANY, bool TWO = false>
FF_D bool ff_traverse_step(const FFBvhView& bvh, FFRayState& r, uint2& cur, FFStack& st)
{
    FFNoCount none;
    return ff_traverse_step<ANY, FFNoCount, TWO>(bvh, r, cur, st, none);
}

// Root group: a fake parent whose only internal child (node 0) sits in the
// slot the ray visits first.
FF_D uint2 ff_root_group(const FFRayState& r)
{
    return make_uint2(0u, (1u << 31) | (1u << (7u ^ r.oct_inv)));
}

// One whole traversal per thread (megakernel paths): closest hit of the ray
// (o, d, [0, inf)), two-sided when `two` (h.prim = -2 - index for a back
// face), or any hit of `ray`; a traversal that exceeds its step bound or
// overflows the stack counts in *err and reports what it found.  Returns
// whether anything was hit.
FF_D bool ff_closest_hit(const FFBvhView& bvh, float3 o, float3 d, FFStack& st, unsigned int* err, ff_hit& h,
                         bool two = false)
{
    FFRayState r;
    ff_ray_setup(r, o, d, two ? -0.f : 0.f, __int_as_float(0x7f800000), false);
    if (bvh.num_nodes) {
        uint2 cur = ff_root_group(r);
        st.reset();
        uint32_t steps = 0;
        while (!ff_traverse_step<false, true>(bvh, r, cur, st)) {
            if (++steps > bvh.num_nodes + 2 || st.overflow) {
                atomicAdd(err, 1u);
                break;
            }
        }
    }
    h = ff_hit_of(r);
    return h.prim != -1;
}

FF_D bool ff_occluded(const FFBvhView& bvh, const ff_ray& ray, FFStack& st, unsigned int* err)
{
    if (!bvh.num_nodes) return false;
    FFRayState r;
    ff_ray_setup(r, make_float3(ray.ox, ray.oy, ray.oz), make_float3(ray.dx, ray.dy, ray.dz), ray.tmin, ray.tmax, true);
    uint2 cur = ff_root_group(r);
    st.reset();
    uint32_t steps = 0;
    while (!ff_traverse_step<true>(bvh, r, cur, st)) {
        if (++steps > bvh.num_nodes + 2 || st.overflow) {
            atomicAdd(err, 1u);
            break;
        }
    }
    return r.prim != 0xffffffffu;
}
