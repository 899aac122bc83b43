// ff_paths.cuh — per-vertex shading of the path tracer, shared by the
// wavefront stages (ff_wavefront.cu) and the path-replay adjoint
// (ff_adjoint.cu): lights (radiance, pdf, visibility ray), the reference's
// mix material (wf_mat_mix + BRDF_L / BRDF_f / BRDF_pdf,
// CUDA-RayTracer/kernel.cu:617-651, dMaterial.cu:363-469), its single-lobe
// stages (wf_mat_diffuse / wf_mat_cook, kernel.cu:546-614) and the two kinds
// without a reference counterpart (thin dielectric, coated diffuse).
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
// (roughness at or above the threshold); a thin dielectric never.
__device__ __forceinline__ bool is_rough(const FFSurf& s, float threshold)
{
    if (s.kind == FF_MAT_DIFFUSE) return true;
    if (s.kind == FF_MAT_DIELECTRIC) return false;
    return s.roughness >= threshold;
}

// wf_mat_mix + BRDF_L / BRDF_f / BRDF_pdf (kernel.cu:617-651, dMaterial.cu:363-469)
__device__ inline void shade_mix(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n, float3 wo,
                          float3 wi, float3 sp, uint32_t key, uint32_t L, ShadeOut& o)
{
    (void)sp;
    const bool corrected = mode == FF_MODE_CORRECTED;
    const float r = mat.roughness;
    float3 Lsum = make_float3(0.f, 0.f, 0.f);
    o.c_nee_ggx = Lsum;
    const float3 Li = light_L(lc, wi);
    const float n_dot_wi = dot3(n, wi);
    if (n_dot_wi > 0.f) {
        const double diff_pdf = diff_get_pdf();
        const double spec_pdf = spec_get_pdf(n, wi, wo, r);
        const double lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        if (lpdf > 0.f && Li != make_float3(0.f, 0.f, 0.f)) {
            // dMaterial.cu:386-393: weights 1 for a delta light
            const double diff_w = lc.is_dir ? 1.0 : power_heuristic(lpdf, diff_pdf);
            const double spec_w = lc.is_dir ? 1.0 : power_heuristic(lpdf, spec_pdf);
            float3 f = spec_f(mat, n, wi, wo) * n_dot_wi;
            if (f != make_float3(0.f, 0.f, 0.f)) Lsum = Lsum + ((f * (float)spec_w) * Li) / (float)lpdf;
            o.c_nee_ggx = Lsum;
            f = diff_f(mat, n, wi, wo) * n_dot_wi;
            if (f != make_float3(0.f, 0.f, 0.f)) Lsum = Lsum + ((f * (float)diff_w) * Li) / (float)lpdf;
        }
    }
    o.c_nee = Lsum;
    const float3 wi_spec = spec_sample(n, wo, r, ff_rand(key, dim_of(L, DIM_SPEC)), ff_rand(key, dim_of(L, DIM_SPEC + 1)));
    const float3 wi_diff = diff_sample(n, ff_rand(key, dim_of(L, DIM_DIFF)), ff_rand(key, dim_of(L, DIM_DIFF + 1)));
    // BSDF-sampled MIS terms (none for a delta light, dMaterial.cu:410);
    // their visibility is traced as shadow rays
    o.ray_spec = o.ray_diff = false;
    if (!lc.is_dir) {
        const float3 org = pos + wi_spec * 0.001f;
        const float nd = dot3(n, wi_spec);
        ff_ray vr;
        if (nd > 0.f && light_vis_ray(lc, org, wi_spec, key, L, DIM_SPEC_VIS, vr)) {
            const double spdf = spec_get_pdf(n, wi_spec, wo, r);
            const double lpdf = light_pdf(lc, pos, wi_spec, key, L, DIM_SPEC_PDF);
            const double wgt = power_heuristic(spdf, lpdf);
            const float3 f = spec_f(mat, n, wi_spec, wo) * nd;
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
            const double dpdf = diff_get_pdf();
            const double lpdf = light_pdf(lc, pos, wi_diff, key, L, DIM_DIFF_PDF);
            const double wgt = power_heuristic(dpdf, lpdf);
            const float3 f = diff_f(mat, n, wi_diff, wo) * nd;
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
    o.ext_f = brdf_f(mat, n, dir, wo);
    o.ext_f_ggx = spec_f(mat, n, dir, wo);
    o.ext_pdf = brdf_pdf(mat, n, dir, wo);
    o.ext_cos = hmax(0.f, dot3(n, dir));
}

// wf_mat_diffuse (kernel.cu:546-577): diff_L returns 0 in the reference (dMaterial.cu:179-227).
__device__ inline void shade_diffuse(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n,
                              float3 wo, float3 wi, uint32_t key, uint32_t L, ShadeOut& o)
{
    o.c_nee = make_float3(0.f, 0.f, 0.f);
    if (mode == FF_MODE_CORRECTED) {
        const float nd = dot3(n, wi);
        const float lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        const float3 Li = light_L(lc, wi);
        if (nd > 0.f && lpdf > 0.f) o.c_nee = ((diff_f(mat, n, wi, wo) * nd) * Li) / lpdf;
    }
    o.ray_spec = o.ray_diff = false;
    const float3 dir = diff_sample(n, ff_rand(key, dim_of(L, DIM_DIFF)), ff_rand(key, dim_of(L, DIM_DIFF + 1)));
    o.ext_d = dir;
    o.ext_f = diff_f(mat, n, dir, wo);
    o.c_nee_ggx = o.ext_f_ggx = make_float3(0.f, 0.f, 0.f);
    o.ext_pdf = (float)diff_get_pdf();
    o.ext_cos = hmax(0.f, dot3(n, dir));
}

// wf_mat_cook (kernel.cu:580-614): spec_L returns 0 in the reference (dMaterial.cu:314-361).
__device__ inline void shade_conductor(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n,
                                float3 wo, float3 wi, uint32_t key, uint32_t L, ShadeOut& o)
{
    o.c_nee = make_float3(0.f, 0.f, 0.f);
    if (mode == FF_MODE_CORRECTED) {
        const float nd = dot3(n, wi);
        const float lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        const float3 Li = light_L(lc, wi);
        if (nd > 0.f && lpdf > 0.f) o.c_nee = ((spec_f(mat, n, wi, wo) * nd) * Li) / lpdf;
    }
    o.ray_spec = o.ray_diff = false;
    const float r = mat.roughness;
    const float3 dir = spec_sample(n, wo, r, ff_rand(key, dim_of(L, DIM_SPEC)), ff_rand(key, dim_of(L, DIM_SPEC + 1)));
    o.ext_d = dir;
    o.ext_f = spec_f(mat, n, dir, wo);
    o.c_nee_ggx = o.c_nee;
    o.ext_f_ggx = o.ext_f;
    o.ext_pdf = spec_get_pdf(n, dir, wo, r);
    o.ext_cos = hmax(0.f, dot3(n, dir));
}

// Thin GGX dielectric (no reference counterpart): with probability equal to
// the Schlick reflectance at the surface's IOR the path reflects off a GGX
// lobe, otherwise it is transmitted through the sheet unchanged.  The
// transmission is a delta lobe (no NEE through it); the GGX reflection gets
// light-sampled NEE.
__device__ inline void shade_dielectric(uint32_t mode, const LightCtx& lc, const FFSurf& mat, float3 pos, float3 n,
                                 float3 wo, float3 wi, uint32_t key, uint32_t L, ShadeOut& o)
{
    (void)mode;
    const float eta = mat.ior > 0.f ? mat.ior : 1.5f;
    const float r0 = ((eta - 1.f) / (eta + 1.f)) * ((eta - 1.f) / (eta + 1.f));
    const float cos_o = fabsf(dot3(n, wo));
    const float x = 1.f - cos_o;
    const float Fr = r0 + (1.f - r0) * x * x * x * x * x;
    FFSurf m = mat;
    m.fresnel = make_float3(r0, r0, r0);
    m.albedo = make_float3(1.f, 1.f, 1.f);
    m.metallic = 0.f;
    o.ray_spec = o.ray_diff = false;
    o.c_nee = make_float3(0.f, 0.f, 0.f);
    const float nd = dot3(n, wi);
    const float lpdf = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
    if (nd > 0.f && lpdf > 0.f) o.c_nee = ((spec_f(m, n, wi, wo) * nd) * light_L(lc, wi)) / lpdf;
    o.c_nee_ggx = o.c_nee;
    if (ff_rand(key, dim_of(L, DIM_EXTRA)) < Fr) {
        const float3 dir = spec_sample(n, wo, m.roughness, ff_rand(key, dim_of(L, DIM_SPEC)),
                                       ff_rand(key, dim_of(L, DIM_SPEC + 1)));
        o.ext_d = dir;
        o.ext_f = spec_f(m, n, dir, wo) / Fr;
        o.ext_f_ggx = o.ext_f;
        o.ext_pdf = spec_get_pdf(n, dir, wo, m.roughness);
        o.ext_cos = hmax(0.f, dot3(n, dir));
    } else {
        const float3 tint = mat.albedo;
        o.ext_d = -wo;
        o.ext_f = tint;
        o.ext_f_ggx = make_float3(0.f, 0.f, 0.f);
        o.ext_pdf = 1.f;
        o.ext_cos = 1.f;
    }
}

// Diffuse base under a GGX clear coat (no reference counterpart): the coat
// reflects with Schlick Fresnel at the coat IOR, the base is Lambertian
// weighted by (1 - F).  Continuation picks the coat lobe or the base with
// equal probability; the pdf is the 50/50 mixture, as BRDF_pdf's.
__device__ inline float3 coat_spec_f(const FFSurf& mat, float3 n, float3 wi, float3 wo, float r0)
{
    FFSurf c = mat;
    c.fresnel = make_float3(r0, r0, r0);
    c.albedo = make_float3(1.f, 1.f, 1.f);
    c.metallic = 0.f;
    return spec_f(c, n, wi, wo);
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
        dir = spec_sample(n, wo, r, ff_rand(key, dim_of(L, DIM_SPEC)), ff_rand(key, dim_of(L, DIM_SPEC + 1)));
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
    o.ext_pdf = 0.5f * spec_get_pdf(n, dir, wo, r) + 0.5f * c * FF_1_PI;
    o.ext_cos = c;
}


}  // namespace ffp
