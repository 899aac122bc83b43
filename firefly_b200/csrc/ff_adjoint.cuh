// ff_adjoint.cuh — pieces of the path-replay adjoint shared by the wavefront
// stages (k_logic / k_shade in adjoint mode, ff_wavefront.cu) and the
// megakernel variants (ff_adjoint.cu): texel footprints, the warp-aggregated
// gradient scatter, and the roughness derivative of one vertex's terms.
// No reference counterpart: the reference renders only.
#pragma once

#include "ff_paths.cuh"

namespace ffadj {

using namespace ffp;

// Bilinear footprint of tex_bilinear (8-bit weights, wrap addressing):
// texel indices and weights.
struct Footprint {
    uint32_t idx[4];
    float w[4];
};
__device__ __forceinline__ Footprint footprint(int w, int h, float u, float v)
{
    float xb = u * (float)w - 0.5f;
    float yb = v * (float)h - 0.5f;
    float fx = floorf(xb), fy = floorf(yb);
    float ax = xb - fx, ay = yb - fy;
    ax = floorf(ax * 256.f + 0.5f) / 256.f;
    ay = floorf(ay * 256.f + 0.5f) / 256.f;
    int ix = (int)fx, iy = (int)fy;
    int x0 = ix % w;
    x0 = x0 < 0 ? x0 + w : x0;
    int x1 = (x0 + 1 == w) ? 0 : x0 + 1;
    int y0 = iy % h;
    y0 = y0 < 0 ? y0 + h : y0;
    int y1 = (y0 + 1 == h) ? 0 : y0 + 1;
    Footprint f;
    f.idx[0] = y0 * w + x0;
    f.idx[1] = y0 * w + x1;
    f.idx[2] = y1 * w + x0;
    f.idx[3] = y1 * w + x1;
    f.w[0] = (1.f - ax) * (1.f - ay);
    f.w[1] = ax * (1.f - ay);
    f.w[2] = (1.f - ax) * ay;
    f.w[3] = ax * ay;
    return f;
}

// Warp-cooperative scatter of a float3 into grad[3*idx .. 3*idx+2]: lanes
// holding the same index are summed first, one lane per distinct index issues
// the atomics.  Returns 1 for the lane that touched the texel.
__device__ __forceinline__ uint32_t scatter_add(float* grad, uint32_t idx, float3 v)
{
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, idx);
    float3 sum = make_float3(0.f, 0.f, 0.f);
    for (uint32_t m = peers; m; m &= m - 1) {
        const int src = __ffs(m) - 1;
        sum.x += __shfl_sync(peers, v.x, src);
        sum.y += __shfl_sync(peers, v.y, src);
        sum.z += __shfl_sync(peers, v.z, src);
    }
    if ((threadIdx.x & 31u) == (uint32_t)(__ffs(peers) - 1)) {
        atomicAdd(grad + 3 * (size_t)idx + 0, sum.x);
        atomicAdd(grad + 3 * (size_t)idx + 1, sum.y);
        atomicAdd(grad + 3 * (size_t)idx + 2, sum.z);
        return 1u;   // one texel touched (12 B of atomics)
    }
    return 0u;
}
__device__ __forceinline__ uint32_t scatter_footprint(float* grad, const Footprint& f, float3 g)
{
    uint32_t n = 0;
#pragma unroll 1
    for (int i = 0; i < 4; ++i) n += scatter_add(grad, f.idx[i], g * f.w[i]);
    return n;
}

// Scalar variant for the roughness channel: adds to grad[3*idx + ch] only.
__device__ __forceinline__ uint32_t scatter_add1(float* grad, uint32_t idx, float v, int ch)
{
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, idx);
    float sum = 0.f;
    for (uint32_t m = peers; m; m &= m - 1) sum += __shfl_sync(peers, v, __ffs(m) - 1);
    if ((threadIdx.x & 31u) == (uint32_t)(__ffs(peers) - 1)) {
        atomicAdd(grad + 3 * (size_t)idx + ch, sum);
        return 1u;
    }
    return 0u;
}
__device__ __forceinline__ uint32_t scatter_footprint1(float* grad, const Footprint& f, float g, int ch)
{
    uint32_t n = 0;
#pragma unroll 1
    for (int i = 0; i < 4; ++i) n += scatter_add1(grad, f.idx[i], g * f.w[i], ch);
    return n;
}

// Which channel of texture `adj` feeds the material's roughness, as
// resolve_surface reads it (get_roughness, dMaterial.cu:25-42): y of the
// packed metallic-roughness texture when the material has one, else x of the
// single-channel roughness texture; -1 when the roughness does not come
// from `adj`.
__device__ __forceinline__ int rough_channel(const ff_material& m, int adj)
{
    if (m.metallic_roughness_tex >= 0) return m.metallic_roughness_tex == adj ? 1 : -1;
    return (m.roughness_tex >= 0 && m.roughness_tex == adj) ? 0 : -1;
}

// Roughness derivative of one vertex's terms (detached sampling: directions,
// pdfs, MIS weights and the roulette stay fixed; only the GGX values D and G
// move with r).  `nee` and `spec` are d/dr of the NEE term c_nee and of the
// mixed material's BSDF-sampled light term c_spec (before the throughput and
// the visibility gate), `dext` is d/dr log(ext_f) per channel: everything the
// path gathers after the vertex carries one factor ext_f.  Each derivative
// is evaluated only where its GGX value is non-zero (0 * NaN would poison the
// sum).  The dielectric's terms are proportional to its D G as well; its
// shading leaves d log(D G)/dr at the NEE and at the sampled direction in
// dlog_nee / dlog_spec (its half vectors differ from ggx_dlog_dr's).
struct RoughTerms {
    float3 nee, spec, dext;
};
__device__ __forceinline__ RoughTerms rough_terms(const ShadeOut& sh, float3 n, float3 wo, float3 wi, float r,
                                                  bool dielectric)
{
    const float3 zero = make_float3(0.f, 0.f, 0.f);
    RoughTerms t;
    t.nee = zero;
    t.spec = zero;
    t.dext = zero;
    if (dielectric) {
        t.nee = sh.c_nee * sh.dlog_nee;
        t.spec = sh.c_spec * sh.dlog_spec;
        if (sh.ext_pdf != 0.f && sh.ext_f != zero) t.dext = make_float3(sh.dlog_spec, sh.dlog_spec, sh.dlog_spec);
        return t;
    }
    // the adjoint runs in corrected mode: the FP32 GGX lobes
    if (sh.c_nee_ggx != zero) t.nee = sh.c_nee_ggx * ggx_dlog_dr32(n, wi, wo, r);
    if (sh.c_spec != zero) {
        const float3 ws = make_float3(sh.r_spec.dx, sh.r_spec.dy, sh.r_spec.dz);
        t.spec = sh.c_spec * ggx_dlog_dr32(n, ws, wo, r);
    }
    if (sh.ext_pdf != 0.f && sh.ext_f_ggx != zero) {
        const float s = ggx_dlog_dr32(n, sh.ext_d, wo, r);
        const float3 df = sh.ext_f_ggx * s;
        t.dext = make_float3(sh.ext_f.x != 0.f ? df.x / sh.ext_f.x : 0.f, sh.ext_f.y != 0.f ? df.y / sh.ext_f.y : 0.f,
                             sh.ext_f.z != 0.f ? df.z / sh.ext_f.z : 0.f);
    }
    return t;
}
// d/dr of the radiance the vertex adds itself, given which of its light
// terms were unoccluded, times the throughput at the vertex.
__device__ __forceinline__ float3 rough_own(const RoughTerms& t, bool vis, bool vis_s, float3 beta)
{
    float3 imm = make_float3(0.f, 0.f, 0.f);
    if (vis) imm = imm + t.nee;
    if (vis_s) imm = imm + t.spec;
    return imm * beta;
}

// dL/d(albedo) per channel of a texture-fed diffuse vertex: everything from
// the vertex on (L_ge = L_s - radiance gathered before it) carries one factor
// of its albedo a.
__device__ __forceinline__ float3 albedo_grad(float3 L_ge, float3 a, float3 dI)
{
    const float3 g = make_float3(a.x > 0.f ? L_ge.x / a.x : 0.f, a.y > 0.f ? L_ge.y / a.y : 0.f,
                                 a.z > 0.f ? L_ge.z / a.z : 0.f);
    return dI * g;
}

}  // namespace ffadj
