// ff_paths.cuh — per-vertex shading of the path tracer, shared by the
// wavefront stages (ff_wavefront.cu) and the path-replay adjoint
// (ff_adjoint.cu): lights (radiance, pdf, visibility ray), the reference's
// mix material (wf_mat_mix + BRDF_L / BRDF_f / BRDF_pdf,
// CUDA-RayTracer/kernel.cu:617-651, dMaterial.cu:363-469), its single-lobe
// stages (wf_mat_diffuse / wf_mat_cook, kernel.cu:546-614) and the two kinds
// without a reference counterpart (rough dielectric, coated diffuse), and the
// rules for paths that run inside refracting objects.
#pragma once

#include "ff_shade.cuh"

namespace ffp {

struct ShadeOut {
    float3 c_nee, c_spec, c_diff;
    // GGX parts of c_nee and ext_f (the terms that depend on the roughness),
    // read by the adjoint only; c_spec, when set, is GGX throughout
    float3 c_nee_ggx, ext_f_ggx;
    bool ray_nee, ray_spec, ray_diff;   // shadow rays to trace
    ff_ray r_nee, r_spec, r_diff;
    float3 ext_o, ext_d, ext_f;
    float ext_pdf, ext_cos;
    // d/dr log f of the dielectric at the NEE direction and at the sampled
    // direction (the adjoint only; the GGX kinds use ggx_dlog_dr instead)
    float dlog_nee, dlog_spec;
};

__device__ __forceinline__ ff_ray make_ray(float3 o, float3 d, float tmax)
{
    return ff_ray{o.x, o.y, o.z, 0.f, d.x, d.y, d.z, tmax};
}

// Light radiance toward wi, pdf of wi, and the visibility ray of light.visible()
// (env and directional: any occluder; area: the rectangle must be hit, and
// the occluder must lie before the projection of a fresh sample point).
// `scale` is the number of lights when one is chosen per vertex (FF_LIGHT_ALL):
// the chosen light's contributions count for all of them.
struct LightCtx {
    FFEnvView env;
    bool is_env;
    bool is_dir;        // dDirectionalLight: delta light
    bool corrected;
    FFRect rect;
    float3 dir, dir_Le;
    float scale;
};

// The lights of a render: -1 env, 0..A-1 area, A..A+D-1 directional,
// FF_LIGHT_ALL one of all (env first when present) per vertex.
struct FFLightSet {
    FFEnvView env;
    bool has_env;
    const ff_area_light* area;
    uint32_t n_area;
    const ff_directional_light* dirs;
    uint32_t n_dir;
    int32_t light;
    bool corrected;
};

__device__ __forceinline__ LightCtx select_light(const FFLightSet& s, uint32_t key, uint32_t L)
{
    LightCtx lc;
    lc.env = s.env;
    lc.corrected = s.corrected;
    lc.is_env = lc.is_dir = false;
    lc.scale = 1.f;
    int32_t id = s.light;
    if (id == FF_LIGHT_ALL) {
        const uint32_t n = (s.has_env ? 1u : 0u) + s.n_area + s.n_dir;
        const uint32_t k = min((uint32_t)(ff_rand(key, dim_of(L, DIM_LIGHT_SEL)) * (float)n), n - 1u);
        lc.scale = (float)n;
        id = s.has_env ? (int32_t)k - 1 : (int32_t)k;
    }
    if (id < 0) {
        lc.is_env = true;
    } else if ((uint32_t)id < s.n_area) {
        lc.rect = make_rect(s.area[id]);
    } else {
        const ff_directional_light& d = s.dirs[(uint32_t)id - s.n_area];
        lc.is_dir = true;
        lc.dir = make_float3(d.direction[0], d.direction[1], d.direction[2]);
        lc.dir_Le = d.radiance * make_float3(d.emissive[0], d.emissive[1], d.emissive[2]);
    }
    return lc;
}

// light.get_direction (kernel.cu:435): the NEE direction and sample point.
__device__ __forceinline__ void sample_light(const LightCtx& lc, float3 pos, uint32_t key, uint32_t L, float3& wi,
                                             float3& sp)
{
    if (lc.is_env) {
        const float ex = ff_rand(key, dim_of(L, DIM_LIGHT)), ey = ff_rand(key, dim_of(L, DIM_LIGHT + 1));
        if (lc.corrected)
            env_sample_corrected(lc.env, pos, ex, ey, ff_rand(key, dim_of(L, DIM_EXTRA + 1)),
                                 ff_rand(key, dim_of(L, DIM_EXTRA + 2)), wi, sp);
        else
            env_sample(lc.env, pos, ex, ey, wi, sp);
    } else if (lc.is_dir) {
        wi = lc.dir;                         // dDirectionalLight::get_direction
        sp = pos;
    } else {
        sp = rect_sample(lc.rect, rand2(key, L, DIM_LIGHT));
        wi = normalize3(sp - pos);
    }
}

__device__ __forceinline__ float3 light_L(const LightCtx& lc, float3 wi)
{
    const float3 Le = lc.is_env ? env_L(lc.env, wi, lc.corrected) : (lc.is_dir ? lc.dir_Le : rect_L(lc.rect, wi));
    return lc.scale == 1.f ? Le : Le * lc.scale;
}
__device__ __forceinline__ float light_pdf(const LightCtx& lc, float3 pos, float3 wi, uint32_t key, uint32_t L,
                                           uint32_t dim)
{
    if (lc.is_env) return lc.corrected ? env_pdf_corrected(lc.env, wi) : env_pdf(lc.env, wi);
    if (lc.is_dir) return 1.f;
    return rect_pdf(lc.rect, pos, rand2(key, L, dim));
}
// Visibility ray of light.visible(ray): returns false when the reference
// answers "not visible" without tracing (area light missed).
__device__ __forceinline__ bool light_vis_ray(const LightCtx& lc, float3 o, float3 d, uint32_t key, uint32_t L,
                                              uint32_t dim, ff_ray& out)
{
    if (lc.is_env || lc.is_dir) {
        out = make_ray(o, d, FF_K_HUGE);
        return true;
    }
    if (!rect_hit(lc.rect, o, d)) return false;
    const float ts = dot3(rect_sample(lc.rect, rand2(key, L, dim)) - o, d);
    out = make_ray(o, d, ts);
    return true;
}

// A vertex where the radiance cache may answer: diffuse, or glossy enough
// (roughness at or above the threshold); a dielectric never.
__device__ __forceinline__ bool is_rough(const FFSurf& s, float threshold)
{
    if (s.kind == FF_MAT_DIFFUSE) return true;
    if (s.kind == FF_MAT_DIELECTRIC) return false;
    return s.roughness >= threshold;
}

// Paths inside refracting objects (no reference counterpart: the reference
// culls back faces, dTriangle.cu:5,41).  A closest hit of a two-sided trace
// reports a back face as prim = -2 - index (ff_hit_of); such a vertex is
// shaded from the inside, with every normal flipped to face the ray.
__device__ __forceinline__ bool hit_back(int32_t prim) { return prim < -1; }
__device__ __forceinline__ uint32_t hit_index(int32_t prim) { return (uint32_t)(prim < -1 ? -2 - prim : prim); }

// The continuation ray of a vertex runs inside an object, and is traced
// two-sided, when the vertex was hit from the inside and the ray stays on
// that side, or when the ray refracts into the object.  side: the sign of
// dot(ext_d, ng), ng facing the incoming ray.
__device__ __forceinline__ bool runs_inside(bool back, bool dielectric, float side)
{
    return back != (dielectric && side < 0.f);
}

// An extension ray; a two-sided one carries the sign bit on tmin (ff_trace.cuh).
__device__ __forceinline__ ff_ray make_ext_ray(float3 o, float3 d, bool two)
{
    return ff_ray{o.x, o.y, o.z, two ? -0.f : 0.f, d.x, d.y, d.z, __int_as_float(0x7f800000)};
}

// wf_mat_mix + BRDF_L / BRDF_f / BRDF_pdf (kernel.cu:617-651, dMaterial.cu:363-469).
// F32 selects the lobe set: the reference's FP64 arithmetic (parity mode) or
// the FP32 restatement (corrected mode), Lobes in ff_shade.cuh.
template <bool F32>
__device__ inline void shade_mix(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n, float3 wo,
                                 float3 wi, float3 sp, uint32_t key, uint32_t L, ShadeOut& o)
{
    using LB = Lobes<F32>;
    using real = typename LB::real;
    (void)sp;
    const bool corrected = mode == FF_MODE_CORRECTED;
    const float r = mat.roughness;
    float3 Lsum = make_float3(0.f, 0.f, 0.f);
    o.c_nee_ggx = Lsum;
    const float3 Li = light_L(lc, wi);
    const float n_dot_wi = dot3(n, wi);
    if (n_dot_wi > 0.f) {
        const real diff_pdf = LB::diff_pdf();
        const real spec_pdf = LB::spec_pdf(n, wi, wo, r);
        const real lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        if (lpdf > 0.f && Li != make_float3(0.f, 0.f, 0.f)) {
            // dMaterial.cu:386-393: weights 1 for a delta light
            const real diff_w = lc.is_dir ? (real)1 : LB::power(lpdf, diff_pdf);
            const real spec_w = lc.is_dir ? (real)1 : LB::power(lpdf, spec_pdf);
            float3 f = LB::spec(mat, n, wi, wo) * n_dot_wi;
            if (f != make_float3(0.f, 0.f, 0.f)) Lsum = Lsum + ((f * (float)spec_w) * Li) / (float)lpdf;
            o.c_nee_ggx = Lsum;
            f = LB::diff(mat, n, wi, wo) * n_dot_wi;
            if (f != make_float3(0.f, 0.f, 0.f)) Lsum = Lsum + ((f * (float)diff_w) * Li) / (float)lpdf;
        }
    }
    o.c_nee = Lsum;
    const float3 wi_spec =
        LB::sample_spec(n, wo, r, ff_rand(key, dim_of(L, DIM_SPEC)), ff_rand(key, dim_of(L, DIM_SPEC + 1)));
    const float3 wi_diff = diff_sample(n, ff_rand(key, dim_of(L, DIM_DIFF)), ff_rand(key, dim_of(L, DIM_DIFF + 1)));
    // BSDF-sampled MIS terms (none for a delta light, dMaterial.cu:410);
    // their visibility is traced as shadow rays
    o.ray_spec = o.ray_diff = false;
    if (!lc.is_dir) {
        const float3 org = pos + wi_spec * 0.001f;
        const float nd = dot3(n, wi_spec);
        ff_ray vr;
        if (nd > 0.f && light_vis_ray(lc, org, wi_spec, key, L, DIM_SPEC_VIS, vr)) {
            const real spdf = LB::spec_pdf(n, wi_spec, wo, r);
            const real lpdf = light_pdf(lc, pos, wi_spec, key, L, DIM_SPEC_PDF);
            const real wgt = LB::power(spdf, lpdf);
            const float3 f = LB::spec(mat, n, wi_spec, wo) * nd;
            const float3 Li2 = light_L(lc, wi_spec);
            if (f != make_float3(0.f, 0.f, 0.f) && spdf > 0.f && Li2 != make_float3(0.f, 0.f, 0.f)) {
                o.c_spec = ((f * Li2) * (float)wgt) / (float)spdf;
                o.ray_spec = true;
                o.r_spec = vr;
            }
        }
    }
    if (!lc.is_dir) {
        // dMaterial.cu:431: the reference offsets this ray along wi_spec (parity)
        const float3 org = corrected ? pos + wi_diff * 0.001f : pos + wi_spec * 0.001f;
        const float nd = dot3(n, wi_diff);
        ff_ray vr;
        if (nd > 0.f && light_vis_ray(lc, org, wi_diff, key, L, DIM_DIFF_VIS, vr)) {
            const real dpdf = LB::diff_pdf();
            const real lpdf = light_pdf(lc, pos, wi_diff, key, L, DIM_DIFF_PDF);
            const real wgt = LB::power(dpdf, lpdf);
            const float3 f = LB::diff(mat, n, wi_diff, wo) * nd;
            const float3 Li2 = light_L(lc, wi_diff);
            if (f != make_float3(0.f, 0.f, 0.f) && dpdf > 0.f && Li2 != make_float3(0.f, 0.f, 0.f)) {
                o.c_diff = ((f * Li2) * (float)wgt) / (float)dpdf;
                o.ray_diff = true;
                o.r_diff = vr;
            }
        }
    }
    const float3 dir = ff_rand(key, dim_of(L, DIM_LOBE)) < 0.5f ? wi_diff : wi_spec;
    o.ext_d = dir;
    // BRDF_f = spec_f + diff_f, BRDF_pdf = 0.5 (spec_pdf + diff_pdf) (dMaterial.cu:459-469)
    o.ext_f_ggx = LB::spec(mat, n, dir, wo);
    o.ext_f = o.ext_f_ggx + LB::diff(mat, n, dir, wo);
    if constexpr (F32) o.ext_pdf = 0.5f * (LB::spec_pdf(n, dir, wo, r) + LB::diff_pdf());
    else o.ext_pdf = (float)(0.5 * (double)(LB::spec_pdf(n, dir, wo, r) + (float)LB::diff_pdf()));
    o.ext_cos = hmax(0.f, dot3(n, dir));
}

// wf_mat_diffuse (kernel.cu:546-577): diff_L returns 0 in the reference (dMaterial.cu:179-227).
template <bool F32>
__device__ inline void shade_diffuse(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n,
                                     float3 wo, float3 wi, uint32_t key, uint32_t L, ShadeOut& o)
{
    using LB = Lobes<F32>;
    o.c_nee = make_float3(0.f, 0.f, 0.f);
    if (mode == FF_MODE_CORRECTED) {
        const float nd = dot3(n, wi);
        const float lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        const float3 Li = light_L(lc, wi);
        if (nd > 0.f && lpdf > 0.f) o.c_nee = ((LB::diff(mat, n, wi, wo) * nd) * Li) / lpdf;
    }
    o.ray_spec = o.ray_diff = false;
    const float3 dir = diff_sample(n, ff_rand(key, dim_of(L, DIM_DIFF)), ff_rand(key, dim_of(L, DIM_DIFF + 1)));
    o.ext_d = dir;
    o.ext_f = LB::diff(mat, n, dir, wo);
    o.c_nee_ggx = o.ext_f_ggx = make_float3(0.f, 0.f, 0.f);
    o.ext_pdf = (float)LB::diff_pdf();
    o.ext_cos = hmax(0.f, dot3(n, dir));
}

// wf_mat_cook (kernel.cu:580-614): spec_L returns 0 in the reference (dMaterial.cu:314-361).
template <bool F32>
__device__ inline void shade_conductor(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n,
                                       float3 wo, float3 wi, uint32_t key, uint32_t L, ShadeOut& o)
{
    using LB = Lobes<F32>;
    o.c_nee = make_float3(0.f, 0.f, 0.f);
    if (mode == FF_MODE_CORRECTED) {
        const float nd = dot3(n, wi);
        const float lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        const float3 Li = light_L(lc, wi);
        if (nd > 0.f && lpdf > 0.f) o.c_nee = ((LB::spec(mat, n, wi, wo) * nd) * Li) / lpdf;
    }
    o.ray_spec = o.ray_diff = false;
    const float r = mat.roughness;
    const float3 dir =
        LB::sample_spec(n, wo, r, ff_rand(key, dim_of(L, DIM_SPEC)), ff_rand(key, dim_of(L, DIM_SPEC + 1)));
    o.ext_d = dir;
    o.ext_f = LB::spec(mat, n, dir, wo);
    o.c_nee_ggx = o.c_nee;
    o.ext_f_ggx = o.ext_f;
    o.ext_pdf = LB::spec_pdf(n, dir, wo, r);
    o.ext_cos = hmax(0.f, dot3(n, dir));
}

// ------------------------------------------------------------ dielectric
// Rough dielectric interface (no reference counterpart; the reference defines
// refract() at dMaterial.cu:97-113 but never calls it).  The BSDF of Walter,
// Marschner, Li and Torrance 2007, "Microfacet models for refraction through
// rough surfaces":
//   D     GGX (their eq. 33) with alpha = r^2, the reference's GGX width
//         (dMaterial.cu:120-125), alpha at least 1e-4;
//   G     Smith shadowing for GGX, G1(wo, h) G1(wi, h) (eq. 34);
//   F     the exact unpolarised Fresnel reflectance of the interface (eq. 22);
//   f_r = F D G / (4 |n.wi| |n.wo|)                                  (eq. 20)
//   f_t = (1 - F) D G |wi.h| |wo.h| eta_o^2
//         / (|n.wi| |n.wo| (eta_o wo.h + eta_t wi.h)^2) * tint       (eq. 21)
// with the radiance scaling (eta_o / eta_t)^2 of a camera path folded into
// f_t, and the transmission tinted by the base colour.  h is the half vector
// of reflection (wi + wo) or refraction (eta_o wo + eta_t wi, eq. 16),
// oriented to the side of n.  Sampling draws a microfacet normal m from
// D(m) |m.n| (eqs. 35-36), then reflects off m with probability F(wo.m) and
// refracts through it otherwise (section 5.3); the pdf of a direction is
// D(h) |h.n| |dh/dwi| times the probability of its branch (eqs. 14, 17).
// wo lies on the side of n, in the medium of index eta_o; eta_t is the
// other side's.  Everything here is FP32.
struct Diel {
    float alpha, eta_o, eta_t;
    float3 tint;
};

// A hit from outside enters the object (eta_o = 1, eta_t = ior); a hit on a
// back face (the ray runs inside) leaves it.
__device__ __forceinline__ Diel diel_of(const FFSurf& m, bool back)
{
    const float ior = m.ior > 0.f ? m.ior : 1.5f;
    Diel d;
    d.alpha = hmax(m.roughness * m.roughness, 1e-4f);
    d.eta_o = back ? ior : 1.f;
    d.eta_t = back ? 1.f : ior;
    d.tint = m.albedo;
    return d;
}

// GGX D(m) for c = n.m (0 for c <= 0).
__device__ __forceinline__ float ggx_d(float alpha, float c)
{
    if (!(c > 0.f)) return 0.f;
    const float a2 = alpha * alpha;
    const float c2 = c * c;
    const float k = c2 * (a2 - 1.f) + 1.f;
    return a2 / ((FF_PI * k) * k);
}

// tan^2 of the angle between v and n, from c = n.v.
__device__ __forceinline__ float tan2_of(float c)
{
    const float c2 = c * c;
    return hmax(0.f, 1.f - c2) / c2;
}

// Smith G1 for GGX: 2 / (1 + sqrt(1 + alpha^2 tan^2)), zero where v sees the
// microfacet from the other side than the macro surface.
__device__ __forceinline__ float smith_g1(float alpha, float vn, float vh)
{
    if (!(vh * vn > 0.f)) return 0.f;
    return 2.f / (1.f + sqrtf(1.f + (alpha * alpha) * tan2_of(vn)));
}

// Fresnel reflectance of a dielectric interface for cos c = wo.m on the
// incident side and relative index n = eta_t / eta_o; 1 under total
// internal reflection.
__device__ __forceinline__ float fresnel_dielectric(float c, float n)
{
    const float g2 = n * n - 1.f + c * c;
    if (g2 < 0.f) return 1.f;
    const float g = sqrtf(g2);
    const float a = (g - c) / (g + c);
    const float b = (c * (g + c) - 1.f) / (c * (g - c) + 1.f);
    return (0.5f * (a * a)) * (1.f + b * b);
}

// Half vector of (wo, wi); false when the pair has none (grazing, or wi on
// the wrong side of the microfacet).
__device__ __forceinline__ bool diel_half(const Diel& d, float3 n, float3 wo, float3 wi, bool& refl, float3& h)
{
    const float cos_o = dot3(n, wo), cos_i = dot3(n, wi);
    if (!(cos_o > 0.f) || cos_i == 0.f) return false;
    refl = cos_i > 0.f;
    if (refl) {
        h = wo + wi;
    } else {
        h = wo * d.eta_o + wi * d.eta_t;
    }
    const float l2 = dot3(h, h);
    if (!(l2 > 0.f)) return false;
    h = normalize3(h);
    if (dot3(h, n) < 0.f) h = -h;
    const float woh = dot3(wo, h), wih = dot3(wi, h);
    if (!(woh > 0.f)) return false;
    return refl ? wih > 0.f : wih < 0.f;
}

// f(wi, wo) and the pdf of sampling wi given wo.
__device__ __forceinline__ void diel_eval(const Diel& d, float3 n, float3 wo, float3 wi, float3& f, float& pdf)
{
    f = make_float3(0.f, 0.f, 0.f);
    pdf = 0.f;
    bool refl;
    float3 h;
    if (!diel_half(d, n, wo, wi, refl, h)) return;
    const float cos_o = dot3(n, wo), cos_i = fabsf(dot3(n, wi));
    const float ch = dot3(n, h), woh = dot3(wo, h), wih = dot3(wi, h);
    const float D = ggx_d(d.alpha, ch);
    const float G = smith_g1(d.alpha, cos_o, woh) * smith_g1(d.alpha, dot3(n, wi), wih);
    const float F = fresnel_dielectric(woh, d.eta_t / d.eta_o);
    if (refl) {
        const float v = ((F * D) * G) / ((4.f * cos_i) * cos_o);
        f = make_float3(v, v, v);
        pdf = ((F * D) * ch) / (4.f * woh);
    } else {
        const float den = d.eta_o * woh + d.eta_t * wih;
        const float den2 = den * den;
        const float v = (((((1.f - F) * D) * G) * (-wih)) * woh * (d.eta_o * d.eta_o)) / ((cos_i * cos_o) * den2);
        f = d.tint * v;
        pdf = ((((1.f - F) * D) * ch) * (d.eta_t * d.eta_t) * (-wih)) / den2;
    }
}

// A microfacet normal drawn from D(m) |m.n| (Walter et al. eqs. 35-36):
// tan^2 theta = alpha^2 e0 / (1 - e0), phi = 2 pi e1, in the frame of n.
__device__ __forceinline__ float3 ggx_sample_normal(float3 n, float alpha, float e0, float e1)
{
    // e0 = 1 (the sampler can return 1.0f) gives t2 = inf: theta = pi / 2
    const float t2 = (alpha * alpha) * (e0 / (1.f - e0));
    const float ct = 1.f / sqrtf(1.f + t2);
    const float st = isinf(t2) ? 1.f : sqrtf(t2) * ct;
    const float phi = FF_2PI * e1;
    float3 T, B;
    frame(n, T, B);
    return normalize3(T * (st * cosf(phi)) + B * (st * sinf(phi)) + n * ct);
}

// The sampled direction (reflection with probability F, else refraction);
// false when the drawn microfacet faces away from wo, or when the reflected
// (refracted) direction ends below (above) the macro surface: diel_eval
// classifies a direction by its side of n, so such a sample has no density
// under the branch that drew it and is dropped (weight 0), as in Walter et
// al.'s sampling.
__device__ __forceinline__ bool diel_sample(const Diel& d, float3 n, float3 wo, float e0, float e1, float e2,
                                            float3& wi)
{
    const float3 m = ggx_sample_normal(n, d.alpha, e0, e1);
    const float woh = dot3(wo, m);
    if (!(woh > 0.f)) return false;
    const float F = fresnel_dielectric(woh, d.eta_t / d.eta_o);
    const bool refl = e2 < F;
    float3 w;
    if (refl) {
        w = m * (2.f * woh) - wo;
    } else {
        const float eta = d.eta_o / d.eta_t;
        const float k = 1.f - (eta * eta) * (1.f - woh * woh);
        w = m * (eta * woh - sqrtf(hmax(k, 0.f))) - wo * eta;
    }
    w = normalize3(w);
    const float c = dot3(n, w);
    if (refl ? !(c > 0.f) : !(c < 0.f)) return false;
    wi = w;
    return true;
}

// d/dr of log(D G) at the pair (wo, wi) (the Fresnel term and the Jacobian
// do not depend on the roughness): with alpha = r^2,
//   dlogD/dalpha = 2 / alpha - 4 alpha c^2 / (c^2 (alpha^2 - 1) + 1)
//   dlogG1/dalpha = -(alpha tan^2 / s) / (1 + s),  s = sqrt(1 + alpha^2 tan^2)
// times dalpha/dr = 2 r (0 where alpha sits at its floor).  The adjoint only.
__device__ __forceinline__ float diel_dlog_dr(const Diel& d, float3 n, float3 wo, float3 wi, float r)
{
    bool refl;
    float3 h;
    if (!diel_half(d, n, wo, wi, refl, h) || !(r * r > 1e-4f)) return 0.f;
    const float a = d.alpha;
    const float c = dot3(n, h), c2 = c * c;
    const float dD = 2.f / a - 4.f * a * c2 / (c2 * (a * a - 1.f) + 1.f);
    float dG = 0.f;
    const float cs[2] = {dot3(n, wo), dot3(n, wi)};
    for (int k = 0; k < 2; ++k) {
        const float t2 = tan2_of(cs[k]);
        const float sq = sqrtf(1.f + a * a * t2);
        dG -= (a * t2 / sq) / (1.f + sq);
    }
    return 2.f * r * (dD + dG);
}

// The dielectric vertex: light-sampled NEE weighted against the BSDF's pdf
// (power heuristic; weight 1 for a delta light), the continuation sampled
// from the BSDF, and, unless the light is a delta light, the light reached
// along the continuation direction weighted against the light's pdf, traced
// as a shadow ray (c_spec / r_spec, as BRDF_L's BSDF-sampled terms).  back:
// the vertex was hit from inside the object.  The NEE shadow ray and the
// continuation leave on the side of their direction (k_shade).
__device__ inline void shade_dielectric(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n,
                                        float3 wo, float3 wi, uint32_t key, uint32_t L, bool back, ShadeOut& o)
{
    (void)mode;
    const Diel d = diel_of(mat, back);
    const float3 zero = make_float3(0.f, 0.f, 0.f);
    o.ray_spec = o.ray_diff = false;
    o.c_nee = o.c_spec = o.c_diff = zero;
    o.dlog_nee = o.dlog_spec = 0.f;
    {
        float3 f;
        float bpdf;
        diel_eval(d, n, wo, wi, f, bpdf);
        const float lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        if (f != zero && lpdf > 0.f) {
            const float w = lc.is_dir ? 1.f : power_heuristic32(lpdf, bpdf);
            o.c_nee = ((f * (fabsf(dot3(n, wi)) * w)) * light_L(lc, wi)) / lpdf;
            o.dlog_nee = diel_dlog_dr(d, n, wo, wi, mat.roughness);
        }
    }
    o.c_nee_ggx = o.c_nee;
    float3 dir = n;
    float3 f = zero;
    float pdf = 0.f;
    if (diel_sample(d, n, wo, ff_rand(key, dim_of(L, DIM_SPEC)), ff_rand(key, dim_of(L, DIM_SPEC + 1)),
                    ff_rand(key, dim_of(L, DIM_EXTRA)), dir))
        diel_eval(d, n, wo, dir, f, pdf);
    else
        dir = n;
    const float c = fabsf(dot3(n, dir));
    if (pdf > 0.f && f != zero) {
        o.dlog_spec = diel_dlog_dr(d, n, wo, dir, mat.roughness);
        ff_ray vr;
        if (!lc.is_dir && light_vis_ray(lc, pos + dir * 0.001f, dir, key, L, DIM_SPEC_VIS, vr)) {
            const float3 Li = light_L(lc, dir);
            if (Li != zero) {
                const float w = power_heuristic32(pdf, light_pdf(lc, pos, dir, key, L, DIM_SPEC_PDF));
                o.c_spec = ((f * (c * w)) * Li) / pdf;
                o.ray_spec = true;
                o.r_spec = vr;
            }
        }
    }
    o.ext_d = dir;
    o.ext_f = f;
    o.ext_f_ggx = f;
    o.ext_pdf = pdf;
    o.ext_cos = c;
}

// Diffuse base under a GGX clear coat (no reference counterpart): the coat
// reflects with Schlick Fresnel at the coat IOR, the base is Lambertian
// weighted by (1 - F).  Continuation picks the coat lobe or the base with
// equal probability; the pdf is the 50/50 mixture, as BRDF_pdf's.  The GGX
// lobe is the reference's spec_f in FP32 (spec_f32): there is no reference
// image of this material to match.
__device__ inline float3 coat_spec_f(const FFSurf& mat, float3 n, float3 wi, float3 wo, float r0)
{
    FFSurf c = mat;
    c.fresnel = make_float3(r0, r0, r0);
    c.albedo = make_float3(1.f, 1.f, 1.f);
    c.metallic = 0.f;
    return spec_f32(c, n, wi, wo);
}
__device__ inline float3 coat_f(const FFSurf& mat, float3 n, float3 wi, float3 wo, float r0)
{
    const float3 spec = coat_spec_f(mat, n, wi, wo, r0);
    const float3 h = normalize3(wo + wi);
    const float x = 1.f - hmax(0.f, dot3(h, wi));
    const float F = r0 + (1.f - r0) * x * x * x * x * x;
    return spec + mat.albedo * ((1.f - F) * FF_1_PI);
}

__device__ inline void shade_coat(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n, float3 wo,
                           float3 wi, uint32_t key, uint32_t L, ShadeOut& o)
{
    (void)mode;
    const float eta = mat.ior > 0.f ? mat.ior : 1.5f;
    const float r0 = ((eta - 1.f) / (eta + 1.f)) * ((eta - 1.f) / (eta + 1.f));
    o.ray_spec = o.ray_diff = false;
    o.c_nee = make_float3(0.f, 0.f, 0.f);
    const float nd = dot3(n, wi);
    const float lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
    o.c_nee_ggx = o.c_nee;
    if (nd > 0.f && lpdf > 0.f) {
        const float3 s = (nd * light_L(lc, wi)) / lpdf;
        o.c_nee = coat_f(mat, n, wi, wo, r0) * s;
        o.c_nee_ggx = coat_spec_f(mat, n, wi, wo, r0) * s;
    }
    const float r = mat.roughness;
    float3 dir;
    if (ff_rand(key, dim_of(L, DIM_LOBE)) < 0.5f) {
        dir = spec_sample32(n, wo, r, ff_rand(key, dim_of(L, DIM_SPEC)), ff_rand(key, dim_of(L, DIM_SPEC + 1)));
    } else {
        // cosine-weighted hemisphere (concentric disk lifted to the hemisphere)
        const float2 dsk = concentric_disk(make_float2(ff_rand(key, dim_of(L, DIM_DIFF)),
                                                       ff_rand(key, dim_of(L, DIM_DIFF + 1))));
        const float z = sqrtf(hmax(0.f, 1.f - dsk.x * dsk.x - dsk.y * dsk.y));
        float3 T, B;
        frame(n, T, B);
        dir = normalize3(T * dsk.x + B * dsk.y + n * z);
    }
    const float c = hmax(0.f, dot3(n, dir));
    o.ext_d = dir;
    o.ext_f = coat_f(mat, n, dir, wo, r0);
    o.ext_f_ggx = coat_spec_f(mat, n, dir, wo, r0);
    o.ext_pdf = 0.5f * spec_get_pdf32(n, dir, wo, r) + 0.5f * c * FF_1_PI;
    o.ext_cos = c;
}


}  // namespace ffp
