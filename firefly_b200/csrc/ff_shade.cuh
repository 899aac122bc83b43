// ff_shade.cuh — materials, lights, camera and sampler of the wavefront path
// tracer, following the reference's arithmetic operation by operation
// (parity mode).  Compiled without FMA contraction (-fmad=false): every float
// expression rounds once per operation in the reference's operand order, and
// every place the reference widens to double (its FP64 GGX terms, MIS
// weights, CDFs) widens here too.
//
// Sources (CUDA-RayTracer/): dMaterial.cu:90-469, dEnvironmentLight.cu:41-103,
// dAreaLight.cu:18-68, Rectangle.cuh:24-123, dCamera.cu:10-36,
// dRandom.cu:49-126, dMath.cuh:1300-1507, Helpers.cu:16-31.
#pragma once

#include "ff_common.cuh"

// ------------------------------------------------------------- dimensions
// Parity sampler: draw d of bounce b of a path sample uses ff_rand(key,
// 32*b + d).  The reference draws from a clock-seeded stream in call order;
// fixing one dimension per call site keeps every draw reproducible even when
// a conditional call site is skipped (the area light's visibility and pdf
// redraws happen only on some branches).  Pairs drawn through
// make_float2(random(), random()) give x the second draw of the pair, the
// order the reference's host build evaluates the arguments in.
enum FFDim : uint32_t {
    DIM_CAM_JITTER = 0,    // 0, 1  UniformSampleSquare in gen_ray
    DIM_CAM_LENS = 2,      // 2, 3  ConcentricSampleDisk in gen_ray
    DIM_LIGHT = 4,         // 4, 5  light get_direction
    DIM_NEE_PDF = 6,       // 6, 7  area light get_pdf redraw in BRDF_L's NEE term
    DIM_SPEC = 8,          // 8, 9  spec_sample e0, e1
    DIM_DIFF = 10,         // 10,11 diff_sample e0, e1
    DIM_SPEC_VIS = 12,     // 12,13 area light visible() redraw, spec MIS ray
    DIM_SPEC_PDF = 14,     // 14,15 area light get_pdf redraw, spec MIS
    DIM_DIFF_VIS = 16,     // 16,17 area light visible() redraw, diff MIS ray
    DIM_DIFF_PDF = 18,     // 18,19 area light get_pdf redraw, diff MIS
    DIM_LOBE = 20,         // 20    random() < 0.5 lobe choice
    DIM_NEE_VIS = 21,      // 21,22 area light visible() redraw of the NEE ray (wf_shadow)
    DIM_RR = 23,           // 23    Russian roulette
    DIM_EXTRA = 24,        // 24..26 materials without a reference counterpart, corrected env jitter
    DIM_LIGHT_SEL = 27     // 27    light choice under FF_LIGHT_ALL
};

FF_D uint32_t dim_of(uint32_t bounce, uint32_t d) { return 32u * bounce + d; }

// UniformSampleSquare / make_float2(random(), random()): x = second draw.
FF_D float2 rand2(uint32_t key, uint32_t bounce, uint32_t d0)
{
    float first = ff_rand(key, dim_of(bounce, d0));
    float second = ff_rand(key, dim_of(bounce, d0 + 1));
    return make_float2(second, first);
}

// ----------------------------------------------------------- vector helpers
// (dMath.cuh) normalize = v * rsqrtf(dot(v, v)); the reference's host build
// defines rsqrtf as 1.0f / sqrtf (dMath.cuh:70-73).
FF_D float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
FF_D float3 cross3(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
FF_D float3 normalize3(float3 v)
{
    float inv = 1.0f / sqrtf(dot3(v, v));
    return v * inv;
}
FF_D float length3(float3 v) { return sqrtf(dot3(v, v)); }
// reflect(i, n) = i - 2.0f * n * dot(n, i)  (dMath.cuh:1402)
FF_D float3 reflect3(float3 i, float3 n) { return i - (2.0f * n) * dot3(n, i); }
// clamp(f, a, b) = fmaxf(a, fminf(f, b)) with the host's a < b ? a : b forms
FF_D float hmin(float a, float b) { return a < b ? a : b; }
FF_D float hmax(float a, float b) { return a > b ? a : b; }
FF_D float clampf(float f, float a, float b) { return hmax(a, hmin(f, b)); }
FF_D float3 lerp3(float3 a, float3 b, float w) { return a * (1.f - w) + b * w; }
// luminance returns (0.299 r + 0.587 g + 0.114 b) evaluated in double, as float (dMath.cuh:1503-1507)
FF_D float luminance(float3 c) { return (float)(0.299 * (double)c.x + 0.587 * (double)c.y + 0.114 * (double)c.z); }
// x^2 and x^5 of the reference's pow(x, 2) / pow(x, 5) (double pow of a widened float)
FF_D double sq_d(double x) { return x * x; }
FF_D double pow5_d(double x)
{
    double x2 = x * x;
    return x2 * x2 * x;
}

// get_orthogonal_vec (dMath.cuh:1450-1463)
FF_D float3 orthogonal_axis(float3 in)
{
    if (fabsf(in.x) < 0.57735026919f) return make_float3(1, 0, 0);
    if (fabsf(in.y) < 0.57735026919f) return make_float3(0, 1, 0);
    return make_float3(0, 0, 1);
}

// sample_spherical_map / sample_spherical_direction (dMath.cuh:1483-1500)
FF_D float2 spherical_map(float3 d)
{
    float2 uv = make_float2(atan2f(d.z, d.x), asinf(d.y));
    uv.x = uv.x * FF_1_2PI;
    uv.y = uv.y * FF_1_PI;
    uv.x = uv.x + 0.5f;
    uv.y = uv.y + 0.5f;
    return uv;
}
FF_D float3 spherical_direction(float2 uv)
{
    float theta = FF_2PI * uv.x;
    float phi = FF_PI * uv.y;
    float x = cosf(theta) * sinf(phi);
    float y = cosf(phi);
    float z = sinf(theta) * sinf(phi);
    return make_float3(-x, -y, -z);
}

// ConcentricSampleDisk(u) (dRandom.cu:83-102)
FF_D float2 concentric_disk(float2 u)
{
    float2 o = make_float2(2.f * u.x - 1.f, 2.f * u.y - 1.f);
    if (o.x == 0 && o.y == 0) return make_float2(0, 0);
    float theta, r;
    if (fabsf(o.x) > fabsf(o.y)) {
        r = o.x;
        theta = FF_PI_4 * (o.y / o.x);
    } else {
        r = o.y;
        theta = FF_PI_2 - FF_PI_4 * (o.x / o.y);
    }
    return make_float2(r * cosf(theta), r * sinf(theta));
}

// -------------------------------------------------------------- materials
struct FFIsect {
    float3 position;
    float3 normal;
    uint32_t material;
    uint32_t prim;
};

// A material resolved at a hit point: the reference's get_albedo /
// get_roughness / get_metallic (dMaterial.cu:10-60) read a texture when one
// is bound, else the factor.
struct FFSurf {
    float3 albedo;
    float3 fresnel;    // dielectric f0
    float roughness;
    float metallic;
    float ior;
    int kind;
};

struct FFTexView {
    const float3* rgb;
    int width, height;
};

// Per-original-triangle tangent frame (the dVertex tangent and bitangent of
// its three vertices), read only at hits on materials with a normal texture.
struct FFTangentTri {
    float3 t0, t1, t2;
    float3 b0, b1, b2;
};

// diff_get_pdf = 1.f / (2.f * M_PI) in float, returned as double (dMaterial.cu:160-163)
FF_D double diff_get_pdf() { return (double)(1.f / (2.f * FF_PI)); }

// fresnel(f0, h, wo) = f0 + (1 - f0) * pow(1 - fmaxf(0, dot(h, wo)), 5) (dMaterial.cu:90-92)
FF_D float3 fresnel3(float3 f0, float3 h, float3 wo)
{
    float x = 1.f - hmax(0.f, dot3(h, wo));
    float p = (float)pow5_d((double)x);
    return f0 + (1.f - f0) * p;
}

// ggxtr_ndf (dMaterial.cu:120-125)
FF_D double ggx_ndf(float3 n, float3 h, float r)
{
    double a2 = r * r * r * r;
    double nh2 = sq_d((double)hmax(0.f, dot3(n, h)));
    return a2 / ((double)FF_PI * sq_d(nh2 * (a2 - 1.0) + 1.0));
}

// geo_atten (dMaterial.cu:126-137); k = powf(r + 1, 2) / 8 in float
FF_D double geo_atten(float3 wi, float3 wo, float3 n, float r)
{
    float rp = r + 1.f;
    double k = (double)((rp * rp) / 8.f);
    double nl = hmax(dot3(n, wi), 0.f);
    double nv = hmax(dot3(n, wo), 0.f);
    double g1 = nl / (nl * (1.0 - k) + k);
    double g2 = nv / (nv * (1.0 - k) + k);
    return g1 * g2;
}

// d/dr of log(D * G) for the GGX lobe of spec_f at roughness r (the Fresnel
// factor and the 4 NoV NoL denominator do not depend on r):
//   D = a2 / (pi (nh2 (a2 - 1) + 1)^2), a2 = r^4:
//       dlogD/dr = 4/r - 8 r^3 nh2 / (nh2 (a2 - 1) + 1)
//   G = g(nl) g(nv), g(x) = x / (x (1 - k) + k), k = (r + 1)^2 / 8:
//       dlogG/dr = -(r + 1)/4 * sum over x in {nl, nv} of (1 - x) / (x (1 - k) + k)
// so that d spec_f / dr = spec_f * ggx_dlog_dr.  Used by the adjoint only.
FF_D double ggx_dlog_dr(float3 n, float3 wi, float3 wo, float r)
{
    const float3 h = normalize3(wo + wi);
    const double rd = (double)r;
    const double a2 = rd * rd * rd * rd;
    const double nh2 = sq_d((double)hmax(0.f, dot3(n, h)));
    const double dlogD = 4.0 / rd - 8.0 * rd * rd * rd * nh2 / (nh2 * (a2 - 1.0) + 1.0);
    const double k = (rd + 1.0) * (rd + 1.0) / 8.0;
    const double nl = hmax(dot3(n, wi), 0.f);
    const double nv = hmax(dot3(n, wo), 0.f);
    const double dlogG = -(rd + 1.0) / 4.0 * ((1.0 - nl) / (nl * (1.0 - k) + k) + (1.0 - nv) / (nv * (1.0 - k) + k));
    return dlogD + dlogG;
}

// power_heuristic(1, f, 1, g) (dMaterial.cu:114-119)
FF_D double power_heuristic(double f, double g) { return (f * f) / (f * f + g * g); }

FF_D float3 f0_of(const FFSurf& m, float3 albedo) { return lerp3(m.fresnel, albedo, m.metallic); }

// diff_f (dMaterial.cu:164-178)
FF_D float3 diff_f(const FFSurf& mat, float3 n, float3 wi, float3 wo)
{
    (void)n;
    float m = mat.metallic;
    float3 a = mat.albedo;
    float3 f0 = f0_of(mat, a);
    float3 wh = normalize3(wo + wi);
    float3 F = fresnel3(f0, wh, wi);
    float3 kd = make_float3(1.f, 1.f, 1.f) - F;
    kd = kd * (float)(1.0 - (double)m);
    return (kd * a) * FF_1_PI;
}

// spec_get_pdf (dMaterial.cu:255-265), returned as float
FF_D float spec_get_pdf(float3 n, float3 wi, float3 wo, float r)
{
    float3 wh = normalize3(wo + wi);
    double wh_dot_n = hmax(dot3(wh, n), 0.f);
    double wo_dot_wh = hmax(dot3(wo, wh), 0.f);
    double D = ggx_ndf(n, wh, r);
    return (float)((D * wh_dot_n) / (double)hmax((float)(4.0 * wo_dot_wh), 0.001f));
}

// spec_f (dMaterial.cu:266-288)
FF_D float3 spec_f(const FFSurf& mat, float3 n, float3 wi, float3 wo)
{
    float r = mat.roughness;
    float3 a = mat.albedo;
    float3 f0 = f0_of(mat, a);
    float3 wh = normalize3(wo + wi);
    double n_dot_wi = hmax(dot3(n, wi), 0.f);
    double n_dot_wo = hmax(dot3(n, wo), 0.f);
    double D = ggx_ndf(n, wh, r);
    double G = geo_atten(wi, wo, n, r);
    float3 F = fresnel3(f0, wh, wi);
    float3 num = (float)(D * G) * F;
    return num / hmax((float)(4.0 * n_dot_wo * n_dot_wi), 0.001f);
}

// Orthonormal frame of the sampling routines: T = normalize(cross(N, axis)), B = normalize(cross(N, T)).
FF_D void frame(float3 N, float3& T, float3& B)
{
    T = normalize3(cross3(N, orthogonal_axis(N)));
    B = normalize3(cross3(N, T));
}

// diff_sample (dMaterial.cu:139-159): uniform hemisphere around N
FF_D float3 diff_sample(float3 N, float e0, float e1)
{
    float sin_theta = sqrtf(1.f - e0 * e0);
    float phi = 2.f * FF_PI * e1;
    float x = sin_theta * cosf(phi);
    float z = sin_theta * sinf(phi);
    float3 T, B;
    frame(N, T, B);
    return normalize3(T * x + N * e0 + B * z);
}

// spec_sample (dMaterial.cu:229-254): GGX half vector, theta and phi in double
FF_D float3 spec_sample(float3 N, float3 wo, float r, float e0, float e1)
{
    double theta = (double)atanf(r * r * sqrtf(e0 / (1.f - e0)));
    double phi = (double)(2 * FF_PI * e1);
    float3 h = make_float3((float)(sin(theta) * cos(phi)), (float)cos(theta), (float)(sin(theta) * sin(phi)));
    float3 T, B;
    frame(N, T, B);
    float3 s = T * h.x + N * h.y + B * h.z;
    return -reflect3(wo, normalize3(s));
}

// BRDF_f = spec_f + diff_f; BRDF_pdf = 0.5 (spec_pdf + diff_pdf) (dMaterial.cu:459-469)
FF_D float3 brdf_f(const FFSurf& m, float3 n, float3 wi, float3 wo)
{
    return spec_f(m, n, wi, wo) + diff_f(m, n, wi, wo);
}
FF_D float brdf_pdf(const FFSurf& m, float3 n, float3 wi, float3 wo)
{
    float sp = spec_get_pdf(n, wi, wo, m.roughness);
    float dp = (float)diff_get_pdf();
    return (float)(0.5 * (double)(sp + dp));
}

// ------------------------------------------------ FP32 lobes (corrected mode)
// The same lobes with every intermediate in FP32.  The reference widens the
// GGX D and G terms, the Fresnel power, the sampling angles and the MIS
// weights to double (dMaterial.cu:114-313); parity mode keeps that, so that
// images match the reference's, while corrected mode, which has no reference
// counterpart to match, computes them in FP32 (the FP64 units of the SM are
// a fraction of its FP32 units, and doubles take two registers each).  Same
// formulas and operand order; the GGX sample takes cos and sin of theta from
// tan(theta) = r^2 sqrt(e0 / (1 - e0)) instead of going through atan.
FF_D float ggx_ndf32(float3 n, float3 h, float r)
{
    const float a2 = r * r * r * r;
    const float nh = hmax(0.f, dot3(n, h));
    const float k = (nh * nh) * (a2 - 1.f) + 1.f;
    return a2 / (FF_PI * (k * k));
}
FF_D float geo_atten32(float3 wi, float3 wo, float3 n, float r)
{
    const float rp = r + 1.f;
    const float k = (rp * rp) / 8.f;
    const float nl = hmax(dot3(n, wi), 0.f);
    const float nv = hmax(dot3(n, wo), 0.f);
    return (nl / (nl * (1.f - k) + k)) * (nv / (nv * (1.f - k) + k));
}
FF_D float3 fresnel32(float3 f0, float3 h, float3 wo)
{
    const float x = 1.f - hmax(0.f, dot3(h, wo));
    const float x2 = x * x;
    const float p = (x2 * x2) * x;
    return f0 + (1.f - f0) * p;
}
FF_D float spec_get_pdf32(float3 n, float3 wi, float3 wo, float r)
{
    const float3 wh = normalize3(wo + wi);
    const float whn = hmax(dot3(wh, n), 0.f);
    const float wowh = hmax(dot3(wo, wh), 0.f);
    return (ggx_ndf32(n, wh, r) * whn) / hmax(4.f * wowh, 0.001f);
}
FF_D float3 spec_f32(const FFSurf& mat, float3 n, float3 wi, float3 wo)
{
    const float r = mat.roughness;
    const float3 f0 = f0_of(mat, mat.albedo);
    const float3 wh = normalize3(wo + wi);
    const float ndwi = hmax(dot3(n, wi), 0.f);
    const float ndwo = hmax(dot3(n, wo), 0.f);
    const float3 F = fresnel32(f0, wh, wi);
    const float3 num = (ggx_ndf32(n, wh, r) * geo_atten32(wi, wo, n, r)) * F;
    return num / hmax((4.f * ndwo) * ndwi, 0.001f);
}
FF_D float3 diff_f32(const FFSurf& mat, float3 n, float3 wi, float3 wo)
{
    (void)n;
    const float3 a = mat.albedo;
    const float3 wh = normalize3(wo + wi);
    float3 kd = make_float3(1.f, 1.f, 1.f) - fresnel32(f0_of(mat, a), wh, wi);
    kd = kd * (1.f - mat.metallic);
    return (kd * a) * FF_1_PI;
}
FF_D float3 spec_sample32(float3 N, float3 wo, float r, float e0, float e1)
{
    // e0 = 1 (the sampler can return 1.0f) gives t = inf: theta = pi / 2
    const float t = (r * r) * sqrtf(e0 / (1.f - e0));
    const float ct = 1.f / sqrtf(1.f + t * t);
    const float st = isinf(t) ? 1.f : t * ct;
    const float phi = FF_2PI * e1;
    float3 T, B;
    frame(N, T, B);
    const float3 s = T * (st * cosf(phi)) + N * ct + B * (st * sinf(phi));
    return -reflect3(wo, normalize3(s));
}
FF_D float power_heuristic32(float f, float g)
{
    const float f2 = f * f;
    return f2 / (f2 + g * g);
}
// d/dr log(D G) of the FP32 GGX lobe (ggx_dlog_dr's derivation).
FF_D float ggx_dlog_dr32(float3 n, float3 wi, float3 wo, float r)
{
    const float3 h = normalize3(wo + wi);
    const float a2 = r * r * r * r;
    const float nh = hmax(0.f, dot3(n, h));
    const float nh2 = nh * nh;
    const float dlogD = 4.f / r - 8.f * r * r * r * nh2 / (nh2 * (a2 - 1.f) + 1.f);
    const float k = (r + 1.f) * (r + 1.f) / 8.f;
    const float nl = hmax(dot3(n, wi), 0.f);
    const float nv = hmax(dot3(n, wo), 0.f);
    return dlogD - (r + 1.f) / 4.f * ((1.f - nl) / (nl * (1.f - k) + k) + (1.f - nv) / (nv * (1.f - k) + k));
}

// The lobe set of a mode: Lobes<false> the reference's (FP64 where it is
// FP64: parity mode), Lobes<true> the FP32 restatement (corrected mode).
template <bool F32>
struct Lobes;
template <>
struct Lobes<false> {
    using real = double;
    static FF_D double diff_pdf() { return diff_get_pdf(); }
    static FF_D float spec_pdf(float3 n, float3 wi, float3 wo, float r) { return spec_get_pdf(n, wi, wo, r); }
    static FF_D float3 spec(const FFSurf& m, float3 n, float3 wi, float3 wo) { return spec_f(m, n, wi, wo); }
    static FF_D float3 diff(const FFSurf& m, float3 n, float3 wi, float3 wo) { return diff_f(m, n, wi, wo); }
    static FF_D float3 sample_spec(float3 n, float3 wo, float r, float e0, float e1)
    {
        return spec_sample(n, wo, r, e0, e1);
    }
    static FF_D double power(double f, double g) { return power_heuristic(f, g); }
    static FF_D float dlog_dr(float3 n, float3 wi, float3 wo, float r) { return (float)ggx_dlog_dr(n, wi, wo, r); }
};
template <>
struct Lobes<true> {
    using real = float;
    static FF_D float diff_pdf() { return 1.f / (2.f * FF_PI); }
    static FF_D float spec_pdf(float3 n, float3 wi, float3 wo, float r) { return spec_get_pdf32(n, wi, wo, r); }
    static FF_D float3 spec(const FFSurf& m, float3 n, float3 wi, float3 wo) { return spec_f32(m, n, wi, wo); }
    static FF_D float3 diff(const FFSurf& m, float3 n, float3 wi, float3 wo) { return diff_f32(m, n, wi, wo); }
    static FF_D float3 sample_spec(float3 n, float3 wo, float r, float e0, float e1)
    {
        return spec_sample32(n, wo, r, e0, e1);
    }
    static FF_D float power(float f, float g) { return power_heuristic32(f, g); }
    static FF_D float dlog_dr(float3 n, float3 wi, float3 wo, float r) { return ggx_dlog_dr32(n, wi, wo, r); }
};

// ----------------------------------------------------------------- lights
// Environment light with importance tables (dEnvironmentLight.cu).
template <class T>
FF_D float3 tex_bilinear(const T* texels, int w, int h, float u, float v);

FF_D FFSurf resolve_surface(const ff_material& m, const FFTexView* tex, float2 uv)
{
    FFSurf s;
    s.albedo = make_float3(m.base_color[0], m.base_color[1], m.base_color[2]);
    if (m.base_color_tex >= 0) {
        const FFTexView t = tex[m.base_color_tex];
        s.albedo = tex_bilinear(t.rgb, t.width, t.height, uv.x, uv.y);
    }
    // get_roughness / get_metallic (dMaterial.cu:25-60): the packed glTF
    // metallic-roughness texture first (roughness in y, metallic in z), then
    // the single-channel textures (x), then the factors
    s.roughness = m.roughness;
    s.metallic = m.metallic;
    if (m.metallic_roughness_tex >= 0) {
        const FFTexView t = tex[m.metallic_roughness_tex];
        const float3 c = tex_bilinear(t.rgb, t.width, t.height, uv.x, uv.y);
        s.roughness = hmax(c.y, 0.01f);
        s.metallic = c.z;
    } else {
        if (m.roughness_tex >= 0) {
            const FFTexView t = tex[m.roughness_tex];
            s.roughness = hmax(tex_bilinear(t.rgb, t.width, t.height, uv.x, uv.y).x, 0.01f);
        }
        if (m.metallic_tex >= 0) {
            const FFTexView t = tex[m.metallic_tex];
            s.metallic = tex_bilinear(t.rgb, t.width, t.height, uv.x, uv.y).x;
        }
    }
    s.fresnel = make_float3(m.fresnel[0], m.fresnel[1], m.fresnel[2]);
    s.ior = m.ior;
    s.kind = m.kind;
    return s;
}
// get_normal (dMaterial.cu:61-88): without a normal texture the interpolated
// normal n; with one, the tangent and bitangent interpolated as the normal is
// (dTriangle::hit, dTriangle.cu:94-96) and n form the frame TBN, the texel c
// becomes q = c * 2 - 1, and the normal is normalize(TBN * q) with the
// reference's Matrix4x4 * float3 (dMatrix.cuh:70-78): q.x T + q.y B + q.z N
// summed in that order, plus the zero translation, over w = 1.
FF_D float3 shading_normal(const ff_material& m, const FFTexView* tex, const FFTangentTri* tan, uint32_t prim,
                           float u, float v, float2 uv, float3 n)
{
    if (m.normal_tex < 0 || !tan) return n;
    const FFTangentTri& f = tan[prim];
    const float3 T = normalize3(u * f.t1 + v * f.t2 + ((1.f - u) - v) * f.t0);
    const float3 B = normalize3(u * f.b1 + v * f.b2 + ((1.f - u) - v) * f.b0);
    const FFTexView t = tex[m.normal_tex];
    const float3 c = tex_bilinear(t.rgb, t.width, t.height, uv.x, uv.y);
    const float3 q = make_float3(c.x * 2.f - 1.f, c.y * 2.f - 1.f, c.z * 2.f - 1.f);
    const float3 o = make_float3(((T.x * q.x + B.x * q.y) + n.x * q.z) + 0.f, ((T.y * q.x + B.y * q.y) + n.y * q.z) + 0.f,
                                 ((T.z * q.x + B.z * q.y) + n.z * q.z) + 0.f);
    const float w = ((0.f * q.x + 0.f * q.y) + 0.f * q.z) + 1.f;
    return normalize3(make_float3(o.x / w, o.y / w, o.z / w));
}

// Guide tables of the CDF searches (built with the tables, ff_envmap.cu):
// for a list of n sorted entries and G buckets, entry k (0 <= k <= G) is
// upper_bound of k / G, the first index whose entry exceeds k / G.  A value v
// in [k / G, (k + 1) / G] has its upper_bound between entries k and k + 1,
// so the search starts from that range instead of [0, n) and ends at the
// same index (upper_bound is monotone in v).  A list that is not sorted
// (or holds a NaN) has every entry kGuideFull: its searches run over [0, n).
constexpr int kGuideMarginal = 1024;   // buckets of the marginal CDF
constexpr int kGuideCond = 512;        // buckets of each conditional row
constexpr uint32_t kGuideFull = 0x80000000u;

struct FFEnvView {
    const float3* rgb;       // width*height texels, row y = v * height
    const double* marginal;  // marginal_y[height]
    const double* cond;      // conds_y[height][width] row-major
    const uint32_t* guide_m;  // kGuideMarginal + 1 entries, or nullptr
    const uint32_t* guide_c;  // height rows of kGuideCond + 1 entries, or nullptr
    const float* pdf;        // pdf texels, already scaled by w*h/(2 pi^2)
    int width, height;
    float3 color;            // constant colour when rgb == nullptr
    float radius;            // 10000 (dEnvironmentLight.cu:14)
    // the same texels and pdf packed as (r, g, b, pdf), or nullptr: one
    // aligned 16-B load per texel, a bilinear pair in one 32-B sector, and
    // the pdf texel of a direction among the four texels of its bilinear
    // lookup (shared cache lines for light_L + light_pdf of one direction)
    const float4* texel4;
};

// tex2DLod<float4> with normalised coordinates, wrap addressing and linear
// filtering: x_B = x*W - 0.5, i = floor(x_B), alpha = frac(x_B) with 8
// fractional bits, as the CUDA Programming Guide specifies texture filtering.
FF_D float3 texel3(const float3* t, int i) { return t[i]; }
FF_D float3 texel3(const float4* t, int i)
{
    const float4 v = t[i];
    return make_float3(v.x, v.y, v.z);
}
template <class T>
FF_D float3 tex_bilinear(const T* texels, int w, int h, float u, float v)
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
    float3 t00 = texel3(texels, y0 * w + x0), t10 = texel3(texels, y0 * w + x1);
    float3 t01 = texel3(texels, y1 * w + x0), t11 = texel3(texels, y1 * w + x1);
    float w00 = (1.f - ax) * (1.f - ay), w10 = ax * (1.f - ay), w01 = (1.f - ax) * ay, w11 = ax * ay;
    return make_float3(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
                       w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
                       w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z);
}

// upper_bound (Helpers.cu:16-31), including its list[left <= val] index.
// With a guide table (see kGuideFull) the search starts from the bucket's
// range; the index it ends at, and so the result, is the full search's.
template <int G = 0>
FF_D int upper_bound_ref(const double* list, int size, float val, const uint32_t* guide = nullptr)
{
    int left = 0, right = size;
    if (G > 0 && guide && val >= 0.f && val <= 1.f) {
        // val * G is exact (G a power of two), so k / G <= val <= (k + 1) / G
        const int k = min((int)(val * (float)G), G - 1);
        const uint32_t a = guide[k], b = guide[k + 1];
        if (!(a & kGuideFull)) {
            left = (int)a;
            right = (int)b;
        }
    }
    while (left < right) {
        int middle = (right - left) / 2 + left;
        if ((double)val >= list[middle]) left = middle + 1;
        else right = middle;
    }
    if (left < size && list[(left <= val) ? 1 : 0] != 0.0) left++;
    return left;
}

// dEnvironmentLight::L (dEnvironmentLight.cu:60-72).  A normalised direction
// can carry a component one ulp above 1, where asinf returns NaN; the
// reference keeps that NaN (parity), corrected mode clamps it.
FF_D float3 env_L(const FFEnvView& e, float3 wi, bool corrected = false)
{
    if (!e.rgb) return e.color;
    if (corrected) wi.y = clampf(wi.y, -1.f, 1.f);
    float2 uv = spherical_map(wi);
    if (e.texel4) return tex_bilinear(e.texel4, e.width, e.height, uv.x, uv.y);
    return tex_bilinear(e.rgb, e.width, e.height, uv.x, uv.y);
}

FF_D const uint32_t* guide_row(const FFEnvView& e, int y)
{
    return e.guide_c ? e.guide_c + (size_t)y * (kGuideCond + 1) : nullptr;
}

// get_direction (dEnvironmentLight.cu:41-58); ex = first draw, ey = second.
FF_D void env_sample(const FFEnvView& e, float3 pos, float ex, float ey, float3& wi, float3& sp)
{
    int y = (int)((float)upper_bound_ref<kGuideMarginal>(e.marginal, e.height, ey, e.guide_m) - 1.f);
    y = y < 0 ? 0 : (y >= e.height ? e.height - 1 : y);
    int x = (int)((float)upper_bound_ref<kGuideCond>(e.cond + (size_t)y * e.width, e.width, ex, guide_row(e, y)) - 1.f);
    x = x < 0 ? 0 : (x >= e.width ? e.width - 1 : x);
    float u = (float)x / (float)e.width;
    float v = (float)y / (float)e.height;
    float3 dir = spherical_direction(make_float2(u, v));
    sp = make_float3(0.f, 0.f, 0.f) + dir * e.radius;
    wi = normalize3(sp - pos);
}

// Corrected-mode environment sampling (no reference counterpart): the texel
// picked from the same CDFs is sampled uniformly and mapped with the inverse
// of spherical_map, so the sampled direction looks up the texel it came
// from; the pdf uses that mapping's Jacobian, cos(latitude) = sqrt(1 - y^2).
// The reference maps the texel corner through sample_spherical_direction
// (a different parametrisation) and divides by sin(acos(wi.z)).
FF_D void env_sample_corrected(const FFEnvView& e, float3 pos, float ex, float ey, float jx, float jy, float3& wi,
                               float3& sp)
{
    int y = (int)((float)upper_bound_ref<kGuideMarginal>(e.marginal, e.height, ey, e.guide_m) - 1.f);
    y = y < 0 ? 0 : (y >= e.height ? e.height - 1 : y);
    int x = (int)((float)upper_bound_ref<kGuideCond>(e.cond + (size_t)y * e.width, e.width, ex, guide_row(e, y)) - 1.f);
    x = x < 0 ? 0 : (x >= e.width ? e.width - 1 : x);
    const float u = ((float)x + jx) / (float)e.width;
    const float v = ((float)y + jy) / (float)e.height;
    const float phi = (u - 0.5f) * FF_2PI;
    const float lat = (v - 0.5f) * FF_PI;
    const float cl = cosf(lat);
    wi = make_float3(cl * cosf(phi), sinf(lat), cl * sinf(phi));
    sp = pos + wi * e.radius;
}
FF_D float env_pdf_corrected(const FFEnvView& e, float3 wi)
{
    float2 uv = spherical_map(wi);
    int x = (int)(uv.x * (float)e.width);
    int y = (int)(uv.y * (float)e.height);
    x = x < 0 ? 0 : (x >= e.width ? e.width - 1 : x);
    y = y < 0 ? 0 : (y >= e.height ? e.height - 1 : y);
    const float cl = sqrtf(hmax(0.f, 1.f - wi.y * wi.y));
    const size_t i = (size_t)y * e.width + x;
    return cl > 0.f ? (e.texel4 ? e.texel4[i].w : e.pdf[i]) / cl : 0.f;
}

// get_pdf(isect, wi) (dEnvironmentLight.cu:83-103): pdf texel over sin(acos(wi.z))
FF_D float env_pdf(const FFEnvView& e, float3 wi)
{
    float2 uv = spherical_map(wi);
    int x = (int)(uv.x * (float)(e.width - 1));
    int y = (int)(uv.y * (float)(e.height - 1));
    float p = 0.f;
    if (x >= 0 && y >= 0 && x < e.width && y < e.height) {
        const size_t i = (size_t)y * e.width + x;
        p = e.texel4 ? e.texel4[i].w : e.pdf[i];
    }
    return p / sinf(acosf(clampf(wi.z, -1.f, 1.f)));
}

// Rectangle area light (Rectangle.cuh, dAreaLight.cu)
struct FFRect {
    float3 p0, a, b, n;
    float a_len2, b_len2, inv_area;
    float3 Le;  // radiance * emissiveColorFactor
};

FF_D FFRect make_rect(const ff_area_light& L)
{
    FFRect r;
    r.p0 = make_float3(L.p0[0], L.p0[1], L.p0[2]);
    r.a = make_float3(L.a[0], L.a[1], L.a[2]);
    r.b = make_float3(L.b[0], L.b[1], L.b[2]);
    r.n = make_float3(L.normal[0], L.normal[1], L.normal[2]);
    float la = length3(r.a), lb = length3(r.b);
    r.a_len2 = la * la;
    r.b_len2 = lb * lb;
    r.inv_area = 1.f / (la * lb);
    r.Le = L.radiance * make_float3(L.emissive[0], L.emissive[1], L.emissive[2]);
    return r;
}

// _Rectangle::sample with u = UniformSampleSquare()
FF_D float3 rect_sample(const FFRect& r, float2 u) { return r.p0 + u.x * r.a + u.y * r.b; }

// _Rectangle::hit(ray) (Rectangle.cuh:74-97)
FF_D bool rect_hit(const FFRect& r, float3 o, float3 d)
{
    float t = dot3(r.p0 - o, r.n) / dot3(d, r.n);
    float3 p = o + t * d;
    float3 p0p = p - r.p0;
    if (t <= FF_K_EPSILON) return false;
    float pa = dot3(p0p, r.a);
    if (pa < 0.0f || pa > r.a_len2) return false;
    float pb = dot3(p0p, r.b);
    if (pb < 0.0f || pb > r.b_len2) return false;
    return true;
}

// dAreaLight::L (dAreaLight.cu:26-34)
FF_D float3 rect_L(const FFRect& r, float3 wi)
{
    float nd = dot3(-r.n, wi);
    return nd > 0.0f ? r.Le : make_float3(0.f, 0.f, 0.f);
}

// dAreaLight::get_pdf(isect, wi) (dAreaLight.cu:47-57): a freshly drawn point
FF_D float rect_pdf(const FFRect& r, float3 pos, float2 u)
{
    float3 sp = rect_sample(r, u);
    float3 w = normalize3(sp - pos);
    float nd = fabsf(dot3(r.n, -w));
    float dist = length3(sp - pos);
    float d2 = dist * dist;
    return (d2 / nd) * r.inv_area;
}

// --------------------------------------------------------------- camera
// dCamera::gen_ray (dCamera.cu:10-36); the NDC is computed in double because
// the reference adds the double literal 0.5 to the pixel coordinate.
FF_D float4 mat_mul4(const float* m, float4 v)
{
    // Matrix4x4 * float4 (dMatrix.cuh:61-69): out.c = sum_i m[i][c] * v_i
    return make_float4(m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12] * v.w,
                       m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13] * v.w,
                       m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14] * v.w,
                       m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15] * v.w);
}

FF_D void gen_camera_ray(const ff_camera& cam, int hres, int vres, int px, int py, float2 jitter, float2 lens,
                         float3& o, float3& d)
{
    float ndx = (float)(2.f * (((double)px + 0.5) / hres) - 1.f);
    float ndy = (float)(1.f - 2.f * (((double)py + 0.5) / vres));
    float4 pn = mat_mul4(cam.inv_view_proj, make_float4(ndx, ndy, -1.f, 1.f));
    float4 pf = mat_mul4(cam.inv_view_proj, make_float4(ndx, ndy, 1.f, 1.f));
    float3 p_near = make_float3(pn.x / pn.w, pn.y / pn.w, pn.z / pn.w);
    float3 p_far = make_float3(pf.x / pf.w, pf.y / pf.w, pf.z / pf.w);
    float2 sp = make_float2(jitter.x * cam.pixel_jitter, jitter.y * cam.pixel_jitter);
    o = p_near + make_float3(sp.x, sp.y, 0.f);
    d = normalize3(p_far - p_near);
    if (cam.lens_radius > 0.f) {
        float3 focal = o + d * cam.focal_distance;
        float2 pl = concentric_disk(lens);
        pl = make_float2(pl.x * cam.lens_radius, pl.y * cam.lens_radius);
        o = o + make_float3(pl.x, pl.y, 0.f);
        d = normalize3(focal - o);
    }
}
