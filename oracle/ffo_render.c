/*
 * ffo_render.c — CPU restatement of the reference's wavefront path tracer,
 * one path sample at a time.  TEST INFRASTRUCTURE ONLY (see ffo.h).
 * Compile with -ffp-contract=off.
 *
 * Follows CUDA-RayTracer/:
 *   wf_logic      kernel.cu:298-455   wf_generate  kernel.cu:458-485
 *   wf_extend     kernel.cu:488-523   wf_shadow    kernel.cu:526-543
 *   wf_mat_mix    kernel.cu:617-651   BRDF_L / BRDF_f / BRDF_pdf dMaterial.cu:363-469
 *   wf_mat_diffuse kernel.cu:546-577  wf_mat_cook  kernel.cu:580-614
 *   lobes         dMaterial.cu:90-313 lights dEnvironmentLight.cu:41-103, dAreaLight.cu:18-68,
 *                                      Rectangle.cuh:74-123
 *   camera        dCamera.cu:10-36    sampler warps dRandom.cu:49-126
 *   env tables    kernel.cu:65-149    upper_bound Helpers.cu:16-31
 * with the reference's clock-seeded random() replaced by the seeded
 * per-(pixel, sample) stream ffo_rand(key, 32 * bounce + site): one fixed
 * dimension per call site (sites listed in ffo.h), x of a make_float2
 * (random(), random()) pair taking the second draw of the pair.
 * Intersections are brute force over all triangles (ffo_trace.c).
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "ffo.h"

#define K_EPS 1e-6f
#define K_HUGE 1e32f
#define PI_F 3.14159265358979323846f
#define TWO_PI_F 6.28318530717958647692f
#define PI_2_F 1.57079632679489661923f
#define PI_4_F 0.785398163397448309615f
#define INV_PI_F 0.318309886183790671537f
#define INV_2PI_F 0.159154943091895335768f

typedef struct { float x, y, z; } v3;

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline v3 mul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 muls(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 smul(float s, v3 a) { return V(s * a.x, s * a.y, s * a.z); }
static inline v3 divs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static inline v3 ssub(float s, v3 a) { return V(s - a.x, s - a.y, s - a.z); }
static inline int iszero(v3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
/* normalize: v * rsqrtf(dot(v,v)), host rsqrtf = 1.0f / sqrtf (dMath.cuh:70-73, 1300-1304) */
static inline v3 normalize(v3 v) { float inv = 1.0f / sqrtf(dot(v, v)); return muls(v, inv); }
static inline float length(v3 v) { return sqrtf(dot(v, v)); }
/* reflect (dMath.cuh:1402) */
static inline v3 reflect(v3 i, v3 n) { return sub(i, muls(smul(2.0f, n), dot(n, i))); }
/* host fminf/fmaxf of dMath.cuh:40-48 */
static inline float hmin(float a, float b) { return a < b ? a : b; }
static inline float hmax(float a, float b) { return a > b ? a : b; }
static inline float clampf_(float f, float a, float b) { return hmax(a, hmin(f, b)); }
static inline v3 lerp3(v3 a, v3 b, float w) { return add(muls(a, 1.f - w), muls(b, w)); }
static inline double sq(double x) { return x * x; }
static inline double pow5(double x) { double x2 = x * x; return x2 * x2 * x; }
static inline v3 ld3(const float* p) { return V(p[0], p[1], p[2]); }

/* ----------------------------------------------------------- sampler */
enum {
    DIM_CAM_JITTER = 0, DIM_CAM_LENS = 2, DIM_LIGHT = 4, DIM_NEE_PDF = 6, DIM_SPEC = 8, DIM_DIFF = 10,
    DIM_SPEC_VIS = 12, DIM_SPEC_PDF = 14, DIM_DIFF_VIS = 16, DIM_DIFF_PDF = 18, DIM_LOBE = 20,
    DIM_NEE_VIS = 21, DIM_RR = 23, DIM_EXTRA = 24, DIM_LIGHT_SEL = 27
};
static inline float R(uint32_t key, uint32_t b, uint32_t d) { return ffo_rand(key, 32u * b + d); }
typedef struct { float x, y; } v2;
static inline v2 R2(uint32_t key, uint32_t b, uint32_t d)
{
    float first = R(key, b, d), second = R(key, b, d + 1);
    v2 r = {second, first};
    return r;
}

static v3 orthogonal_axis(v3 in)
{
    if (fabsf(in.x) < 0.57735026919f) return V(1, 0, 0);
    if (fabsf(in.y) < 0.57735026919f) return V(0, 1, 0);
    return V(0, 0, 1);
}
static void frame(v3 N, v3* T, v3* B)
{
    *T = normalize(cross(N, orthogonal_axis(N)));
    *B = normalize(cross(N, *T));
}
static v2 spherical_map(v3 d)
{
    v2 uv = {atan2f(d.z, d.x), asinf(d.y)};
    uv.x = uv.x * INV_2PI_F;
    uv.y = uv.y * INV_PI_F;
    uv.x = uv.x + 0.5f;
    uv.y = uv.y + 0.5f;
    return uv;
}
static v3 spherical_direction(v2 uv)
{
    float theta = TWO_PI_F * uv.x, phi = PI_F * uv.y;
    float x = cosf(theta) * sinf(phi), y = cosf(phi), z = sinf(theta) * sinf(phi);
    return V(-x, -y, -z);
}
static v2 concentric_disk(v2 u)
{
    v2 o = {2.f * u.x - 1.f, 2.f * u.y - 1.f};
    v2 zero = {0, 0};
    if (o.x == 0 && o.y == 0) return zero;
    float theta, r;
    if (fabsf(o.x) > fabsf(o.y)) { r = o.x; theta = PI_4_F * (o.y / o.x); }
    else { r = o.y; theta = PI_2_F - PI_4_F * (o.x / o.y); }
    v2 out = {r * cosf(theta), r * sinf(theta)};
    return out;
}

/* ---------------------------------------------------------- materials */
static double diff_get_pdf(void) { return (double)(1.f / (2.f * PI_F)); }
static v3 fresnel3(v3 f0, v3 h, v3 wo)
{
    float x = 1.f - hmax(0.f, dot(h, wo));
    float p = (float)pow5((double)x);
    return add(f0, muls(ssub(1.f, f0), p));
}
static double ggx_ndf(v3 n, v3 h, float r)
{
    double a2 = r * r * r * r;
    double nh2 = sq((double)hmax(0.f, dot(n, h)));
    return a2 / ((double)PI_F * sq(nh2 * (a2 - 1.0) + 1.0));
}
static double geo_atten(v3 wi, v3 wo, v3 n, float r)
{
    float rp = r + 1.f;
    double k = (double)((rp * rp) / 8.f);
    double nl = hmax(dot(n, wi), 0.f), nv = hmax(dot(n, wo), 0.f);
    double g1 = nl / (nl * (1.0 - k) + k), g2 = nv / (nv * (1.0 - k) + k);
    return g1 * g2;
}
static double power_heuristic(double f, double g) { return (f * f) / (f * f + g * g); }
/* a material resolved at a hit point (get_albedo / get_roughness, dMaterial.cu:10-43) */
typedef struct { v3 albedo; v3 fresnel; float roughness, metallic, ior; int kind; } surf_t;
static v3 f0_of(const surf_t* m, v3 a) { return lerp3(m->fresnel, a, m->metallic); }
static v3 diff_f(const surf_t* mat, v3 wi, v3 wo)
{
    float m = mat->metallic;
    v3 a = mat->albedo;
    v3 f0 = f0_of(mat, a);
    v3 wh = normalize(add(wo, wi));
    v3 F = fresnel3(f0, wh, wi);
    v3 kd = sub(V(1.f, 1.f, 1.f), F);
    kd = muls(kd, (float)(1.0 - (double)m));
    return muls(mul(kd, a), INV_PI_F);
}
static float spec_get_pdf(v3 n, v3 wi, v3 wo, float r)
{
    v3 wh = normalize(add(wo, wi));
    double whn = hmax(dot(wh, n), 0.f), wowh = hmax(dot(wo, wh), 0.f);
    double D = ggx_ndf(n, wh, r);
    return (float)((D * whn) / (double)hmax((float)(4.0 * wowh), 0.001f));
}
static v3 spec_f(const surf_t* mat, v3 n, v3 wi, v3 wo)
{
    float r = mat->roughness;
    v3 a = mat->albedo;
    v3 f0 = f0_of(mat, a);
    v3 wh = normalize(add(wo, wi));
    double ndwi = hmax(dot(n, wi), 0.f), ndwo = hmax(dot(n, wo), 0.f);
    double D = ggx_ndf(n, wh, r), G = geo_atten(wi, wo, n, r);
    v3 F = fresnel3(f0, wh, wi);
    v3 num = smul((float)(D * G), F);
    return divs(num, hmax((float)(4.0 * ndwo * ndwi), 0.001f));
}
static v3 diff_sample(v3 N, float e0, float e1)
{
    float st = sqrtf(1.f - e0 * e0), phi = 2.f * PI_F * e1;
    float x = st * cosf(phi), z = st * sinf(phi);
    v3 T, B;
    frame(N, &T, &B);
    return normalize(add(add(muls(T, x), muls(N, e0)), muls(B, z)));
}
static v3 spec_sample(v3 N, v3 wo, float r, float e0, float e1)
{
    double theta = (double)atanf(r * r * sqrtf(e0 / (1.f - e0)));
    double phi = (double)(2 * PI_F * e1);
    v3 h = V((float)(sin(theta) * cos(phi)), (float)cos(theta), (float)(sin(theta) * sin(phi)));
    v3 T, B;
    frame(N, &T, &B);
    v3 s = add(add(muls(T, h.x), muls(N, h.y)), muls(B, h.z));
    return neg(reflect(wo, normalize(s)));
}
static v3 brdf_f(const surf_t* m, v3 n, v3 wi, v3 wo) { return add(spec_f(m, n, wi, wo), diff_f(m, wi, wo)); }
static float brdf_pdf(const surf_t* m, v3 n, v3 wi, v3 wo)
{
    float sp = spec_get_pdf(n, wi, wo, m->roughness);
    float dp = (float)diff_get_pdf();
    return (float)(0.5 * (double)(sp + dp));
}

/* FP32 lobes of the corrected mode (the product's Lobes<true>,
 * firefly_b200/csrc/ff_shade.cuh): the same formulas and operand order with
 * every intermediate in float; the GGX sample takes cos and sin of theta
 * from tan(theta) = r^2 sqrt(e0 / (1 - e0)).  Parity mode keeps the
 * reference's FP64 (the functions above). */
static float ggx_ndf32(v3 n, v3 h, float r)
{
    float a2 = r * r * r * r;
    float nh = hmax(0.f, dot(n, h));
    float k = (nh * nh) * (a2 - 1.f) + 1.f;
    return a2 / (PI_F * (k * k));
}
static float geo_atten32(v3 wi, v3 wo, v3 n, float r)
{
    float rp = r + 1.f;
    float k = (rp * rp) / 8.f;
    float nl = hmax(dot(n, wi), 0.f), nv = hmax(dot(n, wo), 0.f);
    return (nl / (nl * (1.f - k) + k)) * (nv / (nv * (1.f - k) + k));
}
static v3 fresnel32(v3 f0, v3 h, v3 wo)
{
    float x = 1.f - hmax(0.f, dot(h, wo));
    float x2 = x * x;
    float p = (x2 * x2) * x;
    return add(f0, muls(ssub(1.f, f0), p));
}
static float spec_get_pdf32(v3 n, v3 wi, v3 wo, float r)
{
    v3 wh = normalize(add(wo, wi));
    float whn = hmax(dot(wh, n), 0.f), wowh = hmax(dot(wo, wh), 0.f);
    return (ggx_ndf32(n, wh, r) * whn) / hmax(4.f * wowh, 0.001f);
}
static v3 spec_f32(const surf_t* mat, v3 n, v3 wi, v3 wo)
{
    float r = mat->roughness;
    v3 f0 = f0_of(mat, mat->albedo);
    v3 wh = normalize(add(wo, wi));
    float ndwi = hmax(dot(n, wi), 0.f), ndwo = hmax(dot(n, wo), 0.f);
    v3 F = fresnel32(f0, wh, wi);
    v3 num = smul(ggx_ndf32(n, wh, r) * geo_atten32(wi, wo, n, r), F);
    return divs(num, hmax((4.f * ndwo) * ndwi, 0.001f));
}
static v3 diff_f32(const surf_t* mat, v3 wi, v3 wo)
{
    v3 a = mat->albedo;
    v3 wh = normalize(add(wo, wi));
    v3 kd = sub(V(1.f, 1.f, 1.f), fresnel32(f0_of(mat, a), wh, wi));
    kd = muls(kd, 1.f - mat->metallic);
    return muls(mul(kd, a), INV_PI_F);
}
static v3 spec_sample32(v3 N, v3 wo, float r, float e0, float e1)
{
    float t = (r * r) * sqrtf(e0 / (1.f - e0));   /* e0 = 1: t = inf, theta = pi / 2 */
    float ct = 1.f / sqrtf(1.f + t * t);
    float st = isinf(t) ? 1.f : t * ct;
    float phi = TWO_PI_F * e1;
    v3 T, B;
    frame(N, &T, &B);
    v3 s = add(add(muls(T, st * cosf(phi)), muls(N, ct)), muls(B, st * sinf(phi)));
    return neg(reflect(wo, normalize(s)));
}
static float diff_pdf32(void) { return 1.f / (2.f * PI_F); }

/* ------------------------------------------------------------- lights */
/* luminance (dMath.cuh:1503-1507): double arithmetic, float result */
static float luminance(v3 c) { return (float)(0.299 * (double)c.x + 0.587 * (double)c.y + 0.114 * (double)c.z); }

/* tex2DLod, linear filter, wrap, normalised coords, 8 fractional weight bits */
static v3 tex_bilinear(const float* rgb, int w, int h, float u, float v)
{
    float xb = u * (float)w - 0.5f, yb = v * (float)h - 0.5f;
    float fx = floorf(xb), fy = floorf(yb);
    float ax = xb - fx, ay = yb - fy;
    ax = floorf(ax * 256.f + 0.5f) / 256.f;
    ay = floorf(ay * 256.f + 0.5f) / 256.f;
    int ix = (int)fx, iy = (int)fy;
    int x0 = ix % w; x0 = x0 < 0 ? x0 + w : x0;
    int x1 = (x0 + 1 == w) ? 0 : x0 + 1;
    int y0 = iy % h; y0 = y0 < 0 ? y0 + h : y0;
    int y1 = (y0 + 1 == h) ? 0 : y0 + 1;
    const float *t00 = rgb + 3 * (y0 * w + x0), *t10 = rgb + 3 * (y0 * w + x1);
    const float *t01 = rgb + 3 * (y1 * w + x0), *t11 = rgb + 3 * (y1 * w + x1);
    float w00 = (1.f - ax) * (1.f - ay), w10 = ax * (1.f - ay), w01 = (1.f - ax) * ay, w11 = ax * ay;
    return V(w00 * t00[0] + w10 * t10[0] + w01 * t01[0] + w11 * t11[0],
             w00 * t00[1] + w10 * t10[1] + w01 * t01[1] + w11 * t11[1],
             w00 * t00[2] + w10 * t10[2] + w01 * t01[2] + w11 * t11[2]);
}

static int upper_bound_ref(const double* list, int size, float val)
{
    int left = 0, right = size;
    while (left < right) {
        int middle = (right - left) / 2 + left;
        if ((double)val >= list[middle]) left = middle + 1;
        else right = middle;
    }
    if (left < size && list[(left <= val) ? 1 : 0] != 0.0) left++;
    return left;
}

/* The serial table build of kernel.cu:65-149 over the emulated texture. */
void ffo_env_build(const float* rgb, int w, int h, double* marginal, double* cond, float* pdf, double* denom_out)
{
    double denom = 0.0;
    for (int j = 0; j < h; j++) {
        float v = (float)j / (float)h;
        double st = (double)sinf(PI_F * v);
        for (int i = 0; i < w; i++) {
            float u = (float)i / (float)w;
            double lum = luminance(tex_bilinear(rgb, w, h, u, v));
            denom += lum * st;
        }
    }
    double* mp = (double*)malloc(sizeof(double) * (size_t)h);
    for (int j = 0; j < h; j++) {
        float v = (float)j / (float)h;
        double st = (double)sinf(PI_F * v) / denom;
        mp[j] = 0.f;
        for (int i = 0; i < w; i++) {
            float u = (float)i / (float)w;
            double lum = luminance(tex_bilinear(rgb, w, h, u, v));
            mp[j] += lum * st;
        }
        marginal[j] = j ? mp[j] + marginal[j - 1] : mp[j];
    }
    for (int y = 0; y < h; y++) {
        float v = (float)y / (float)h;
        double st = (double)sinf(PI_F * v);
        double val = st / (denom * mp[y]);
        double* row = cond + (size_t)y * w;
        for (int x = 0; x < w; x++) {
            float u = (float)x / (float)w;
            double lum = luminance(tex_bilinear(rgb, w, h, u, v));
            row[x] = lum * val;
            if (x) row[x] += row[x - 1];
        }
    }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            float u = (float)x / (float)w, v = (float)y / (float)h;
            double st = (double)sinf(PI_F * v);
            double lum = luminance(tex_bilinear(rgb, w, h, u, v));
            float p = (float)((lum * st) / denom);
            p *= (float)(w * h) / (2.f * PI_F * PI_F);
            pdf[(size_t)y * w + x] = p;
        }
    if (denom_out) *denom_out = denom;
    free(mp);
}

typedef struct { v3 p0, a, b, n; float a_len2, b_len2, inv_area; v3 Le; } rect_t;

static rect_t make_rect(const ffo_area_light* L)
{
    rect_t r;
    r.p0 = ld3(L->p0); r.a = ld3(L->a); r.b = ld3(L->b); r.n = ld3(L->normal);
    float la = length(r.a), lb = length(r.b);
    r.a_len2 = la * la;
    r.b_len2 = lb * lb;
    r.inv_area = 1.f / (la * lb);
    r.Le = smul(L->radiance, ld3(L->emissive));
    return r;
}
static v3 rect_sample(const rect_t* r, v2 u) { return add(add(r->p0, smul(u.x, r->a)), smul(u.y, r->b)); }
static int rect_hit(const rect_t* r, v3 o, v3 d)
{
    float t = dot(sub(r->p0, o), r->n) / dot(d, r->n);
    v3 p = add(o, smul(t, d));
    v3 p0p = sub(p, r->p0);
    if (t <= K_EPS) return 0;
    float pa = dot(p0p, r->a);
    if (pa < 0.0f || pa > r->a_len2) return 0;
    float pb = dot(p0p, r->b);
    if (pb < 0.0f || pb > r->b_len2) return 0;
    return 1;
}
static v3 rect_L(const rect_t* r, v3 wi) { return dot(neg(r->n), wi) > 0.0f ? r->Le : V(0, 0, 0); }
static float rect_pdf(const rect_t* r, v3 pos, v2 u)
{
    v3 sp = rect_sample(r, u);
    v3 w = normalize(sub(sp, pos));
    float nd = fabsf(dot(r->n, neg(w)));
    float dist = length(sub(sp, pos));
    float d2 = dist * dist;
    return (d2 / nd) * r->inv_area;
}

typedef struct {
    const ffo_render_desc* d;
    int is_env;
    int is_dir;          /* delta light (dDirectionalLight) */
    int corrected;
    rect_t rect;
    v3 dir, dir_Le;
    float scale;         /* number of lights under per-vertex selection, else 1 */
    const double* marginal;
    const double* cond;
    const float* pdf;
} light_ctx;

static v3 env_L(const ffo_render_desc* d, v3 wi)
{
    if (!d->env_rgb) return ld3(d->env_color);
    if (d->mode == 1) wi.y = clampf_(wi.y, -1.f, 1.f);   /* corrected mode: no asinf(>1) NaN */
    v2 uv = spherical_map(wi);
    return tex_bilinear(d->env_rgb, d->env_w, d->env_h, uv.x, uv.y);
}
static float env_pdf(const light_ctx* lc, v3 wi)
{
    const ffo_render_desc* d = lc->d;
    v2 uv = spherical_map(wi);
    int x = (int)(uv.x * (float)(d->env_w - 1)), y = (int)(uv.y * (float)(d->env_h - 1));
    float p = (x >= 0 && y >= 0 && x < d->env_w && y < d->env_h) ? lc->pdf[(size_t)y * d->env_w + x] : 0.f;
    return p / sinf(acosf(clampf_(wi.z, -1.f, 1.f)));
}
static void env_sample(const light_ctx* lc, v3 pos, float ex, float ey, v3* wi, v3* sp)
{
    const ffo_render_desc* d = lc->d;
    int y = (int)((float)upper_bound_ref(lc->marginal, d->env_h, ey) - 1.f);
    y = y < 0 ? 0 : (y >= d->env_h ? d->env_h - 1 : y);
    int x = (int)((float)upper_bound_ref(lc->cond + (size_t)y * d->env_w, d->env_w, ex) - 1.f);
    x = x < 0 ? 0 : (x >= d->env_w ? d->env_w - 1 : x);
    v2 uv = {(float)x / (float)d->env_w, (float)y / (float)d->env_h};
    v3 dir = spherical_direction(uv);
    *sp = add(V(0.f, 0.f, 0.f), muls(dir, 10000.f));
    *wi = normalize(sub(*sp, pos));
}
/* corrected mode: uniform point in the chosen texel, inverse of spherical_map, cos(latitude) Jacobian */
static void env_sample_corrected(const light_ctx* lc, v3 pos, float ex, float ey, float jx, float jy, v3* wi, v3* sp)
{
    const ffo_render_desc* d = lc->d;
    int y = (int)((float)upper_bound_ref(lc->marginal, d->env_h, ey) - 1.f);
    y = y < 0 ? 0 : (y >= d->env_h ? d->env_h - 1 : y);
    int x = (int)((float)upper_bound_ref(lc->cond + (size_t)y * d->env_w, d->env_w, ex) - 1.f);
    x = x < 0 ? 0 : (x >= d->env_w ? d->env_w - 1 : x);
    float u = ((float)x + jx) / (float)d->env_w, v = ((float)y + jy) / (float)d->env_h;
    float phi = (u - 0.5f) * TWO_PI_F, lat = (v - 0.5f) * PI_F;
    float cl = cosf(lat);
    *wi = V(cl * cosf(phi), sinf(lat), cl * sinf(phi));
    *sp = add(pos, muls(*wi, 10000.f));
}
static float env_pdf_corrected(const light_ctx* lc, v3 wi)
{
    const ffo_render_desc* d = lc->d;
    v2 uv = spherical_map(wi);
    int x = (int)(uv.x * (float)d->env_w), y = (int)(uv.y * (float)d->env_h);
    x = x < 0 ? 0 : (x >= d->env_w ? d->env_w - 1 : x);
    y = y < 0 ? 0 : (y >= d->env_h ? d->env_h - 1 : y);
    float cl = sqrtf(hmax(0.f, 1.f - wi.y * wi.y));
    return cl > 0.f ? lc->pdf[(size_t)y * d->env_w + x] / cl : 0.f;
}
static v3 light_L(const light_ctx* lc, v3 wi)
{
    v3 Le = lc->is_env ? env_L(lc->d, wi) : (lc->is_dir ? lc->dir_Le : rect_L(&lc->rect, wi));
    return lc->scale == 1.f ? Le : muls(Le, lc->scale);
}
static float light_pdf(const light_ctx* lc, v3 pos, v3 wi, uint32_t key, uint32_t L, uint32_t dim)
{
    if (lc->is_env) return lc->corrected ? env_pdf_corrected(lc, wi) : env_pdf(lc, wi);
    if (lc->is_dir) return 1.f;
    return rect_pdf(&lc->rect, pos, R2(key, L, dim));
}

typedef struct { v3 o, d; float tmax; } ray_t;

static int light_vis_ray(const light_ctx* lc, v3 o, v3 d, uint32_t key, uint32_t L, uint32_t dim, ray_t* out)
{
    if (lc->is_env || lc->is_dir) { out->o = o; out->d = d; out->tmax = K_HUGE; return 1; }
    if (!rect_hit(&lc->rect, o, d)) return 0;
    float ts = dot(sub(rect_sample(&lc->rect, R2(key, L, dim)), o), d);
    out->o = o; out->d = d; out->tmax = ts;
    return 1;
}

/* ------------------------------------------------------------- tracing */
/* Closest hit over all triangles, ties to the lowest index.  two_sided: a
 * ray inside an object also takes back faces, returned as -2 - index. */
static int closest(const ffo_render_desc* d, v3 o, v3 dir, int two_sided, float* t_out, float* u_out, float* v_out)
{
    float best = K_HUGE, bu = 0, bv = 0;
    int prim = -1;
    const float oo[3] = {o.x, o.y, o.z}, dd[3] = {dir.x, dir.y, dir.z};
    for (int i = 0; i < d->num_tris; ++i) {
        const float* tri = d->tris + 9 * (size_t)i;
        float t, u, v;
        int back = 0;
        int ok = two_sided ? ffo_intersect_two_sided(tri, tri + 3, tri + 6, oo, dd, &t, &u, &v, &back)
                           : ffo_intersect_cull(tri, tri + 3, tri + 6, oo, dd, &t, &u, &v);
        if (ok && !(t < 0) && t < best) {
            best = t; bu = u; bv = v; prim = back ? -2 - i : i;
        }
    }
    *t_out = best; *u_out = bu; *v_out = bv;
    return prim;
}
static int occluded(const ffo_render_desc* d, const ray_t* r)
{
    const float oo[3] = {r->o.x, r->o.y, r->o.z}, dd[3] = {r->d.x, r->d.y, r->d.z};
    for (int i = 0; i < d->num_tris; ++i) {
        const float* tri = d->tris + 9 * (size_t)i;
        float t;
        if (ffo_shadow_hit(tri, tri + 3, tri + 6, oo, dd, &t) && t >= 0.f && t < r->tmax) return 1;
    }
    return 0;
}

/* ------------------------------------------------------------- shading */
typedef struct {
    v3 c_nee, c_spec, c_diff;
    int has_nee, has_spec, has_diff;
    ray_t r_nee, r_spec, r_diff;
    v3 ext_o, ext_d, ext_f;
    float ext_pdf, ext_cos;
} shade_t;

static void shade_mix(const light_ctx* lc, int corrected, const surf_t* mat, v3 pos, v3 n, v3 wo, v3 wi,
                      uint32_t key, uint32_t L, shade_t* o)
{
    float r = mat->roughness;
    v3 Lsum = V(0, 0, 0);
    v3 Li = light_L(lc, wi);
    float ndwi = dot(n, wi);
    if (ndwi > 0.f) {
        double dp = diff_get_pdf();
        double sp = spec_get_pdf(n, wi, wo, r);
        double lp = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        if (lp > 0.f && !iszero(Li)) {
            /* dMaterial.cu:386-393: weights 1 for a delta light */
            double dw = lc->is_dir ? 1.0 : power_heuristic(lp, dp), sw = lc->is_dir ? 1.0 : power_heuristic(lp, sp);
            v3 f = muls(spec_f(mat, n, wi, wo), ndwi);
            if (!iszero(f)) Lsum = add(Lsum, divs(mul(muls(f, (float)sw), Li), (float)lp));
            f = muls(diff_f(mat, wi, wo), ndwi);
            if (!iszero(f)) Lsum = add(Lsum, divs(mul(muls(f, (float)dw), Li), (float)lp));
        }
    }
    o->c_nee = Lsum;
    v3 wi_spec = spec_sample(n, wo, r, R(key, L, DIM_SPEC), R(key, L, DIM_SPEC + 1));
    v3 wi_diff = diff_sample(n, R(key, L, DIM_DIFF), R(key, L, DIM_DIFF + 1));
    o->has_spec = o->has_diff = 0;
    if (!lc->is_dir) {   /* no BSDF-sampled terms for a delta light (dMaterial.cu:410) */
        v3 org = add(pos, muls(wi_spec, 0.001f));
        float nd = dot(n, wi_spec);
        ray_t vr;
        if (nd > 0.f && light_vis_ray(lc, org, wi_spec, key, L, DIM_SPEC_VIS, &vr)) {
            double sp = spec_get_pdf(n, wi_spec, wo, r);
            double lp = light_pdf(lc, pos, wi_spec, key, L, DIM_SPEC_PDF);
            double w = power_heuristic(sp, lp);
            v3 f = muls(spec_f(mat, n, wi_spec, wo), nd);
            v3 Li2 = light_L(lc, wi_spec);
            if (!iszero(f) && sp > 0.f && !iszero(Li2)) {
                o->c_spec = divs(muls(mul(f, Li2), (float)w), (float)sp);
                o->has_spec = 1;
                o->r_spec = vr;
            }
        }
    }
    if (!lc->is_dir) {
        v3 org = corrected ? add(pos, muls(wi_diff, 0.001f)) : add(pos, muls(wi_spec, 0.001f));
        float nd = dot(n, wi_diff);
        ray_t vr;
        if (nd > 0.f && light_vis_ray(lc, org, wi_diff, key, L, DIM_DIFF_VIS, &vr)) {
            double dp = diff_get_pdf();
            double lp = light_pdf(lc, pos, wi_diff, key, L, DIM_DIFF_PDF);
            double w = power_heuristic(dp, lp);
            v3 f = muls(diff_f(mat, wi_diff, wo), nd);
            v3 Li2 = light_L(lc, wi_diff);
            if (!iszero(f) && dp > 0.f && !iszero(Li2)) {
                o->c_diff = divs(muls(mul(f, Li2), (float)w), (float)dp);
                o->has_diff = 1;
                o->r_diff = vr;
            }
        }
    }
    v3 dir = R(key, L, DIM_LOBE) < 0.5f ? wi_diff : wi_spec;
    o->ext_d = dir;
    o->ext_f = brdf_f(mat, n, dir, wo);
    o->ext_pdf = brdf_pdf(mat, n, dir, wo);
    o->ext_cos = hmax(0.f, dot(n, dir));
}

/* shade_mix in corrected mode: the FP32 lobes (the product's shade_mix<true>). */
static float power_heuristic32(float f, float g)
{
    float f2 = f * f;
    return f2 / (f2 + g * g);
}
static void shade_mix32(const light_ctx* lc, const surf_t* mat, v3 pos, v3 n, v3 wo, v3 wi, uint32_t key,
                        uint32_t L, shade_t* o)
{
    float r = mat->roughness;
    v3 Lsum = V(0, 0, 0);
    v3 Li = light_L(lc, wi);
    float ndwi = dot(n, wi);
    if (ndwi > 0.f) {
        float dp = diff_pdf32();
        float sp = spec_get_pdf32(n, wi, wo, r);
        float lp = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        if (lp > 0.f && !iszero(Li)) {
            float dw = lc->is_dir ? 1.f : power_heuristic32(lp, dp), sw = lc->is_dir ? 1.f : power_heuristic32(lp, sp);
            v3 f = muls(spec_f32(mat, n, wi, wo), ndwi);
            if (!iszero(f)) Lsum = add(Lsum, divs(mul(muls(f, sw), Li), lp));
            f = muls(diff_f32(mat, wi, wo), ndwi);
            if (!iszero(f)) Lsum = add(Lsum, divs(mul(muls(f, dw), Li), lp));
        }
    }
    o->c_nee = Lsum;
    v3 wi_spec = spec_sample32(n, wo, r, R(key, L, DIM_SPEC), R(key, L, DIM_SPEC + 1));
    v3 wi_diff = diff_sample(n, R(key, L, DIM_DIFF), R(key, L, DIM_DIFF + 1));
    o->has_spec = o->has_diff = 0;
    if (!lc->is_dir) {
        v3 org = add(pos, muls(wi_spec, 0.001f));
        float nd = dot(n, wi_spec);
        ray_t vr;
        if (nd > 0.f && light_vis_ray(lc, org, wi_spec, key, L, DIM_SPEC_VIS, &vr)) {
            float sp = spec_get_pdf32(n, wi_spec, wo, r);
            float lp = light_pdf(lc, pos, wi_spec, key, L, DIM_SPEC_PDF);
            float w = power_heuristic32(sp, lp);
            v3 f = muls(spec_f32(mat, n, wi_spec, wo), nd);
            v3 Li2 = light_L(lc, wi_spec);
            if (!iszero(f) && sp > 0.f && !iszero(Li2)) {
                o->c_spec = divs(muls(mul(f, Li2), w), sp);
                o->has_spec = 1;
                o->r_spec = vr;
            }
        }
    }
    if (!lc->is_dir) {
        v3 org = add(pos, muls(wi_diff, 0.001f));
        float nd = dot(n, wi_diff);
        ray_t vr;
        if (nd > 0.f && light_vis_ray(lc, org, wi_diff, key, L, DIM_DIFF_VIS, &vr)) {
            float dp = diff_pdf32();
            float lp = light_pdf(lc, pos, wi_diff, key, L, DIM_DIFF_PDF);
            float w = power_heuristic32(dp, lp);
            v3 f = muls(diff_f32(mat, wi_diff, wo), nd);
            v3 Li2 = light_L(lc, wi_diff);
            if (!iszero(f) && dp > 0.f && !iszero(Li2)) {
                o->c_diff = divs(muls(mul(f, Li2), w), dp);
                o->has_diff = 1;
                o->r_diff = vr;
            }
        }
    }
    v3 dir = R(key, L, DIM_LOBE) < 0.5f ? wi_diff : wi_spec;
    o->ext_d = dir;
    v3 fs = spec_f32(mat, n, dir, wo);
    o->ext_f = add(fs, diff_f32(mat, dir, wo));
    o->ext_pdf = 0.5f * (spec_get_pdf32(n, dir, wo, r) + diff_pdf32());
    o->ext_cos = hmax(0.f, dot(n, dir));
}

static void shade_diffuse(const light_ctx* lc, int corrected, const surf_t* mat, v3 pos, v3 n, v3 wo, v3 wi,
                          uint32_t key, uint32_t L, shade_t* o)
{
    o->c_nee = V(0, 0, 0);
    if (corrected) {
        float nd = dot(n, wi);
        float lp = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        v3 Li = light_L(lc, wi);
        if (nd > 0.f && lp > 0.f) o->c_nee = divs(mul(muls(diff_f32(mat, wi, wo), nd), Li), lp);
    }
    o->has_spec = o->has_diff = 0;
    v3 dir = diff_sample(n, R(key, L, DIM_DIFF), R(key, L, DIM_DIFF + 1));
    o->ext_d = dir;
    o->ext_f = corrected ? diff_f32(mat, dir, wo) : diff_f(mat, dir, wo);
    o->ext_pdf = corrected ? diff_pdf32() : (float)diff_get_pdf();
    o->ext_cos = hmax(0.f, dot(n, dir));
}

static void shade_conductor(const light_ctx* lc, int corrected, const surf_t* mat, v3 pos, v3 n, v3 wo, v3 wi,
                            uint32_t key, uint32_t L, shade_t* o)
{
    o->c_nee = V(0, 0, 0);
    if (corrected) {
        float nd = dot(n, wi);
        float lp = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        v3 Li = light_L(lc, wi);
        if (nd > 0.f && lp > 0.f) o->c_nee = divs(mul(muls(spec_f32(mat, n, wi, wo), nd), Li), lp);
    }
    o->has_spec = o->has_diff = 0;
    float r = mat->roughness;
    v3 dir = corrected ? spec_sample32(n, wo, r, R(key, L, DIM_SPEC), R(key, L, DIM_SPEC + 1))
                       : spec_sample(n, wo, r, R(key, L, DIM_SPEC), R(key, L, DIM_SPEC + 1));
    o->ext_d = dir;
    o->ext_f = corrected ? spec_f32(mat, n, dir, wo) : spec_f(mat, n, dir, wo);
    o->ext_pdf = corrected ? spec_get_pdf32(n, dir, wo, r) : spec_get_pdf(n, dir, wo, r);
    o->ext_cos = hmax(0.f, dot(n, dir));
}

/* ---------------------------------------------------------- dielectric
 * Rough dielectric interface (no reference counterpart; the reference's
 * refract(), dMaterial.cu:97-113, is never called), restated from Walter,
 * Marschner, Li and Torrance 2007, "Microfacet models for refraction through
 * rough surfaces", as the product computes it (shade_dielectric,
 * firefly_b200/csrc/ff_paths.cuh), operation for operation in FP32:
 *   D GGX (their eq. 33), alpha = max(r^2, 1e-4); G = G1(wo) G1(wi), Smith
 *   for GGX (eq. 34); F exact unpolarised Fresnel (eq. 22);
 *   f_r = F D G / (4 |n.wi| |n.wo|) (eq. 20);
 *   f_t = (1 - F) D G |wi.h| |wo.h| eta_o^2 / (|n.wi| |n.wo| (eta_o wo.h + eta_t wi.h)^2) * tint (eq. 21,
 *         radiance scaling folded in);
 *   sampling: m from D(m)|m.n| (eqs. 35-36), reflect with probability F,
 *   else refract (section 5.3); pdf = D(h) |h.n| |dh/dwi| x the branch's
 *   probability (eqs. 14, 17). */
typedef struct { float alpha, eta_o, eta_t; v3 tint; } diel_t;

static diel_t diel_of(const surf_t* m, int back)
{
    float ior = m->ior > 0.f ? m->ior : 1.5f;
    diel_t d;
    d.alpha = hmax(m->roughness * m->roughness, 1e-4f);
    d.eta_o = back ? ior : 1.f;
    d.eta_t = back ? 1.f : ior;
    d.tint = m->albedo;
    return d;
}
static float ggx_d(float alpha, float c)
{
    if (!(c > 0.f)) return 0.f;
    float a2 = alpha * alpha;
    float c2 = c * c;
    float k = c2 * (a2 - 1.f) + 1.f;
    return a2 / ((PI_F * k) * k);
}
static float tan2_of(float c)
{
    float c2 = c * c;
    return hmax(0.f, 1.f - c2) / c2;
}
static float smith_g1(float alpha, float vn, float vh)
{
    if (!(vh * vn > 0.f)) return 0.f;
    return 2.f / (1.f + sqrtf(1.f + (alpha * alpha) * tan2_of(vn)));
}
static float fresnel_dielectric(float c, float n)
{
    float g2 = n * n - 1.f + c * c;
    if (g2 < 0.f) return 1.f;
    float g = sqrtf(g2);
    float a = (g - c) / (g + c);
    float b = (c * (g + c) - 1.f) / (c * (g - c) + 1.f);
    return (0.5f * (a * a)) * (1.f + b * b);
}
static int diel_half(const diel_t* d, v3 n, v3 wo, v3 wi, int* refl, v3* h)
{
    float cos_o = dot(n, wo), cos_i = dot(n, wi);
    if (!(cos_o > 0.f) || cos_i == 0.f) return 0;
    *refl = cos_i > 0.f;
    v3 hh = *refl ? add(wo, wi) : add(muls(wo, d->eta_o), muls(wi, d->eta_t));
    float l2 = dot(hh, hh);
    if (!(l2 > 0.f)) return 0;
    hh = normalize(hh);
    if (dot(hh, n) < 0.f) hh = neg(hh);
    *h = hh;
    float woh = dot(wo, hh), wih = dot(wi, hh);
    if (!(woh > 0.f)) return 0;
    return *refl ? wih > 0.f : wih < 0.f;
}
static void diel_eval(const diel_t* d, v3 n, v3 wo, v3 wi, v3* f, float* pdf)
{
    *f = V(0, 0, 0);
    *pdf = 0.f;
    int refl;
    v3 h;
    if (!diel_half(d, n, wo, wi, &refl, &h)) return;
    float cos_o = dot(n, wo), cos_i = fabsf(dot(n, wi));
    float ch = dot(n, h), woh = dot(wo, h), wih = dot(wi, h);
    float D = ggx_d(d->alpha, ch);
    float G = smith_g1(d->alpha, cos_o, woh) * smith_g1(d->alpha, dot(n, wi), wih);
    float F = fresnel_dielectric(woh, d->eta_t / d->eta_o);
    if (refl) {
        float v = ((F * D) * G) / ((4.f * cos_i) * cos_o);
        *f = V(v, v, v);
        *pdf = ((F * D) * ch) / (4.f * woh);
    } else {
        float den = d->eta_o * woh + d->eta_t * wih;
        float den2 = den * den;
        float v = (((((1.f - F) * D) * G) * (-wih)) * woh * (d->eta_o * d->eta_o)) / ((cos_i * cos_o) * den2);
        *f = muls(d->tint, v);
        *pdf = ((((1.f - F) * D) * ch) * (d->eta_t * d->eta_t) * (-wih)) / den2;
    }
}
static v3 ggx_sample_normal(v3 n, float alpha, float e0, float e1)
{
    float t2 = (alpha * alpha) * (e0 / (1.f - e0));   /* e0 = 1: t2 = inf, theta = pi / 2 */
    float ct = 1.f / sqrtf(1.f + t2);
    float st = isinf(t2) ? 1.f : sqrtf(t2) * ct;
    float phi = TWO_PI_F * e1;
    v3 T, B;
    frame(n, &T, &B);
    return normalize(add(add(muls(T, st * cosf(phi)), muls(B, st * sinf(phi))), muls(n, ct)));
}
static int diel_sample(const diel_t* d, v3 n, v3 wo, float e0, float e1, float e2, v3* wi)
{
    v3 m = ggx_sample_normal(n, d->alpha, e0, e1);
    float woh = dot(wo, m);
    if (!(woh > 0.f)) return 0;
    float F = fresnel_dielectric(woh, d->eta_t / d->eta_o);
    int refl = e2 < F;
    v3 w;
    if (refl) {
        w = sub(muls(m, 2.f * woh), wo);
    } else {
        float eta = d->eta_o / d->eta_t;
        float k = 1.f - (eta * eta) * (1.f - woh * woh);
        w = sub(muls(m, eta * woh - sqrtf(hmax(k, 0.f))), muls(wo, eta));
    }
    w = normalize(w);
    /* a reflection below / refraction above the macro surface has no
     * density under its branch (diel_eval classifies by side): dropped */
    float c = dot(n, w);
    if (refl ? !(c > 0.f) : !(c < 0.f)) return 0;
    *wi = w;
    return 1;
}
static float power_heuristic_f(float f, float g)
{
    float f2 = f * f;
    return f2 / (f2 + g * g);
}
static void shade_dielectric(const light_ctx* lc, const surf_t* mat, v3 pos, v3 n, v3 wo, v3 wi, uint32_t key,
                             uint32_t L, int back, shade_t* o)
{
    const diel_t d = diel_of(mat, back);
    o->has_spec = o->has_diff = 0;
    o->c_nee = o->c_spec = o->c_diff = V(0, 0, 0);
    {
        v3 f;
        float bpdf;
        diel_eval(&d, n, wo, wi, &f, &bpdf);
        float lp = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
        if (!iszero(f) && lp > 0.f) {
            float w = lc->is_dir ? 1.f : power_heuristic_f(lp, bpdf);
            o->c_nee = divs(mul(muls(f, fabsf(dot(n, wi)) * w), light_L(lc, wi)), lp);
        }
    }
    v3 dir = n, f = V(0, 0, 0);
    float pdf = 0.f;
    if (diel_sample(&d, n, wo, R(key, L, DIM_SPEC), R(key, L, DIM_SPEC + 1), R(key, L, DIM_EXTRA), &dir))
        diel_eval(&d, n, wo, dir, &f, &pdf);
    else
        dir = n;
    float c = fabsf(dot(n, dir));
    if (pdf > 0.f && !iszero(f)) {
        ray_t vr;
        if (!lc->is_dir && light_vis_ray(lc, add(pos, muls(dir, 0.001f)), dir, key, L, DIM_SPEC_VIS, &vr)) {
            v3 Li = light_L(lc, dir);
            if (!iszero(Li)) {
                float w = power_heuristic_f(pdf, light_pdf(lc, pos, dir, key, L, DIM_SPEC_PDF));
                o->c_spec = divs(mul(muls(f, c * w), Li), pdf);
                o->has_spec = 1;
                o->r_spec = vr;
            }
        }
    }
    o->ext_d = dir;
    o->ext_f = f;
    o->ext_pdf = pdf;
    o->ext_cos = c;
}

/* ----------------------------------------------------------------- coat
 * Diffuse base under a GGX clear coat (no reference counterpart), as the
 * product computes it (shade_coat, firefly_b200/csrc/ff_paths.cuh): the coat
 * is the reference's spec_f (dMaterial.cu:266-288) with f0 = ((ior - 1) /
 * (ior + 1))^2, white albedo and no metal; the base is albedo (1 - F) / pi
 * with Schlick's F at the half vector; light-sampled NEE without MIS; the
 * continuation picks the coat's GGX sample (spec_sample) or a cosine-weighted
 * direction (concentric disk lifted to the hemisphere) with probability 1/2
 * each, pdf the 50/50 mixture. */
static v3 coat_spec_f(const surf_t* mat, v3 n, v3 wi, v3 wo, float r0)
{
    surf_t c = *mat;
    c.fresnel = V(r0, r0, r0);
    c.albedo = V(1.f, 1.f, 1.f);
    c.metallic = 0.f;
    return spec_f32(&c, n, wi, wo);
}
static v3 coat_f(const surf_t* mat, v3 n, v3 wi, v3 wo, float r0)
{
    v3 spec = coat_spec_f(mat, n, wi, wo, r0);
    v3 h = normalize(add(wo, wi));
    float x = 1.f - hmax(0.f, dot(h, wi));
    float F = r0 + (1.f - r0) * x * x * x * x * x;
    return add(spec, muls(mat->albedo, (1.f - F) * INV_PI_F));
}
static void shade_coat(const light_ctx* lc, const surf_t* mat, v3 pos, v3 n, v3 wo, v3 wi, uint32_t key,
                       uint32_t L, shade_t* o)
{
    float eta = mat->ior > 0.f ? mat->ior : 1.5f;
    float r0 = ((eta - 1.f) / (eta + 1.f)) * ((eta - 1.f) / (eta + 1.f));
    o->has_spec = o->has_diff = 0;
    o->c_nee = V(0, 0, 0);
    float nd = dot(n, wi);
    float lp = light_pdf(lc, pos, wi, key, L, DIM_NEE_PDF);
    if (nd > 0.f && lp > 0.f) {
        v3 sc = divs(smul(nd, light_L(lc, wi)), lp);
        o->c_nee = mul(coat_f(mat, n, wi, wo, r0), sc);
    }
    float r = mat->roughness;
    v3 dir;
    if (R(key, L, DIM_LOBE) < 0.5f) {
        dir = spec_sample32(n, wo, r, R(key, L, DIM_SPEC), R(key, L, DIM_SPEC + 1));
    } else {
        v2 u = {R(key, L, DIM_DIFF), R(key, L, DIM_DIFF + 1)};
        v2 dsk = concentric_disk(u);
        float z = sqrtf(hmax(0.f, 1.f - dsk.x * dsk.x - dsk.y * dsk.y));
        v3 T, B;
        frame(n, &T, &B);
        dir = normalize(add(add(muls(T, dsk.x), muls(B, dsk.y)), muls(n, z)));
    }
    float c = hmax(0.f, dot(n, dir));
    o->ext_d = dir;
    o->ext_f = coat_f(mat, n, dir, wo, r0);
    o->ext_pdf = 0.5f * spec_get_pdf32(n, dir, wo, r) + 0.5f * c * INV_PI_F;
    o->ext_cos = c;
}

/* gen_ray (dCamera.cu:10-36); NDC in double because of the 0.5 double literal */
static void camera_ray(const ffo_render_desc* d, int px, int py, v2 jit, v2 lens, v3* o, v3* dir)
{
    const float* m = d->cam_inv;
    float ndx = (float)(2.f * (((double)px + 0.5) / d->width) - 1.f);
    float ndy = (float)(1.f - 2.f * (((double)py + 0.5) / d->height));
    float pn[4], pf[4];
    for (int c = 0; c < 4; ++c) {
        pn[c] = m[c] * ndx + m[4 + c] * ndy + m[8 + c] * -1.f + m[12 + c] * 1.f;
        pf[c] = m[c] * ndx + m[4 + c] * ndy + m[8 + c] * 1.f + m[12 + c] * 1.f;
    }
    v3 p_near = V(pn[0] / pn[3], pn[1] / pn[3], pn[2] / pn[3]);
    v3 p_far = V(pf[0] / pf[3], pf[1] / pf[3], pf[2] / pf[3]);
    v2 sp = {jit.x * d->cam_jitter, jit.y * d->cam_jitter};
    *o = add(p_near, V(sp.x, sp.y, 0.f));
    *dir = normalize(sub(p_far, p_near));
    if (d->cam_lens_radius > 0.f) {
        v3 focal = add(*o, muls(*dir, d->cam_focal));
        v2 pl = concentric_disk(lens);
        pl.x = pl.x * d->cam_lens_radius;
        pl.y = pl.y * d->cam_lens_radius;
        *o = add(*o, V(pl.x, pl.y, 0.f));
        *dir = normalize(sub(focal, *o));
    }
}

/* The light of a vertex: the fixed one, or under light == -2 one of all
 * lights (env first when present, then area, then directional) chosen from
 * the draw DIM_LIGHT_SEL, its contributions scaled by the number of lights. */
static light_ctx select_light(const light_ctx* base, uint32_t key, uint32_t L)
{
    const ffo_render_desc* d = base->d;
    light_ctx lc = *base;
    int id = d->light;
    lc.scale = 1.f;
    if (id == -2) {
        uint32_t n = (d->env_rgb ? 1u : 0u) + (uint32_t)d->num_area_lights + (uint32_t)d->num_dir_lights;
        uint32_t k = (uint32_t)(R(key, L, DIM_LIGHT_SEL) * (float)n);
        if (k > n - 1) k = n - 1;
        lc.scale = (float)n;
        id = d->env_rgb ? (int)k - 1 : (int)k;
    }
    lc.is_env = id < 0;
    lc.is_dir = 0;
    if (id >= 0 && id < d->num_area_lights) {
        lc.rect = make_rect(&d->area_lights[id]);
    } else if (id >= d->num_area_lights) {
        const ffo_dir_light* dl = &d->dir_lights[id - d->num_area_lights];
        double x = dl->direction[0], y = dl->direction[1], z = dl->direction[2];
        double len = sqrt(x * x + y * y + z * z);
        lc.is_dir = 1;
        lc.dir = V((float)(x / len), (float)(y / len), (float)(z / len));
        lc.dir_Le = smul(dl->radiance, ld3(dl->emissive));
    }
    return lc;
}

/* One path sample; returns its radiance (sum of the contributions). */
/* get_albedo / get_roughness / get_metallic (dMaterial.cu:10-60) at texcoord
 * (tu, tv): the base-colour texture; the packed metallic-roughness texture
 * first (roughness y, metallic z), then the roughness / metallic textures
 * (x), then the factors already in sf. */
static void resolve_textures(const ffo_material* mm, const ffo_texture* textures, float tu, float tv, surf_t* sf)
{
    if (mm->base_color_tex >= 0) {
        const ffo_texture* tx = &textures[mm->base_color_tex];
        sf->albedo = tex_bilinear(tx->rgb, tx->width, tx->height, tu, tv);
    }
    if (mm->metallic_roughness_tex >= 0) {
        const ffo_texture* tx = &textures[mm->metallic_roughness_tex];
        v3 c = tex_bilinear(tx->rgb, tx->width, tx->height, tu, tv);
        sf->roughness = hmax(c.y, 0.01f);
        sf->metallic = c.z;
    } else {
        if (mm->roughness_tex >= 0) {
            const ffo_texture* tx = &textures[mm->roughness_tex];
            sf->roughness = hmax(tex_bilinear(tx->rgb, tx->width, tx->height, tu, tv).x, 0.01f);
        }
        if (mm->metallic_tex >= 0) {
            const ffo_texture* tx = &textures[mm->metallic_tex];
            sf->metallic = tex_bilinear(tx->rgb, tx->width, tx->height, tu, tv).x;
        }
    }
}

/* get_normal (dMaterial.cu:61-88) under a normal texture: texel c mapped to
 * q = c * 2 - 1, then the Matrix4x4(T, B, N) * float3 product of
 * dMatrix.cuh:70-78: ((T q.x + B q.y) + N q.z) + 0 over w = ((0 + 0) + 0) + 1,
 * normalised. */
static v3 normal_from_map(v3 T, v3 B, v3 N, v3 c)
{
    v3 q = {c.x * 2.f - 1.f, c.y * 2.f - 1.f, c.z * 2.f - 1.f};
    v3 o3 = {((T.x * q.x + B.x * q.y) + N.x * q.z) + 0.f, ((T.y * q.x + B.y * q.y) + N.y * q.z) + 0.f,
             ((T.z * q.x + B.z * q.y) + N.z * q.z) + 0.f};
    float w3 = ((0.f * q.x + 0.f * q.y) + 0.f * q.z) + 1.f;
    v3 r = {o3.x / w3, o3.y / w3, o3.z / w3};
    return normalize(r);
}

static void path_sample(const ffo_render_desc* d, const light_ctx* lc_base, int px, int py, uint32_t sample,
                        double out[3], uint64_t* n_ext, uint64_t* n_sh)
{
    const int corrected = d->mode == 1;
    uint32_t pixel = (uint32_t)(py * d->width + px);
    uint32_t key = ffo_path_key(d->seed, pixel, sample);
    v3 o, dir;
    camera_ray(d, px, py, R2(key, 0, DIM_CAM_JITTER), R2(key, 0, DIM_CAM_LENS), &o, &dir);
    v3 beta = V(1, 1, 1);
    uint32_t L = 0;
    shade_t sh;
    memset(&sh, 0, sizeof(sh));
    int vis_nee = 0, vis_spec = 0, vis_diff = 0;
    int inside = 0;   /* the ray runs inside an object: two-sided closest hit */
    out[0] = out[1] = out[2] = 0.0;
    for (;;) {
        float t, u, v;
        int hit = closest(d, o, dir, inside, &t, &u, &v);
        (*n_ext)++;
        L += 1;
        int found = hit != -1;
        int back = hit < -1;   /* a back face: the vertex is shaded from the inside */
        int prim = back ? -2 - hit : hit;
        int terminate = (L > (uint32_t)d->max_depth) || !found;
        if (!found && L == 1) {
            v3 c = mul(beta, env_L(d, dir));
            out[0] += c.x; out[1] += c.y; out[2] += c.z;
        }
        if (L > 1) {
            if (corrected) {
                if (vis_nee || vis_spec || vis_diff) {
                    v3 lb = V(0, 0, 0);
                    if (vis_nee) lb = add(lb, sh.c_nee);
                    if (vis_spec) lb = add(lb, sh.c_spec);
                    if (vis_diff) lb = add(lb, sh.c_diff);
                    v3 c = mul(lb, beta);
                    out[0] += c.x; out[1] += c.y; out[2] += c.z;
                }
            } else if (vis_nee) {
                v3 lb = sh.c_nee;
                if (sh.has_spec && vis_spec) lb = add(lb, sh.c_spec);
                if (sh.has_diff && vis_diff) lb = add(lb, sh.c_diff);
                v3 c = mul(lb, beta);
                out[0] += c.x; out[1] += c.y; out[2] += c.z;
            }
            if (iszero(sh.ext_f) || sh.ext_pdf == 0.f) {
                terminate = 1;
            } else {
                beta = mul(beta, divs(muls(sh.ext_f, sh.ext_cos), sh.ext_pdf));
                if (L > (uint32_t)d->rr_depth) {
                    float q = hmax(0.05f, 1.f - beta.y);
                    if (R(key, L, DIM_RR) < q) terminate = 1;
                    else if (corrected) {
                        if (q >= 1.f) terminate = 1;
                        else beta = divs(beta, 1.f - q);
                    }
                }
            }
        }
        if (terminate) break;
        /* hit attributes (dTriangle::hit) */
        const float* nn = d->normals + 9 * (size_t)prim;
        v3 n0 = ld3(nn), n1 = ld3(nn + 3), n2 = ld3(nn + 6);
        v3 n = normalize(add(add(smul(u, n1), smul(v, n2)), smul((1.f - u) - v, n0)));
        v3 pos = add(o, smul(t, dir));
        v3 wi, sp;
        const light_ctx lcv = select_light(lc_base, key, L);
        const light_ctx* lc = &lcv;
        if (lc->is_env) {
            if (corrected)
                env_sample_corrected(lc, pos, R(key, L, DIM_LIGHT), R(key, L, DIM_LIGHT + 1), R(key, L, DIM_EXTRA + 1),
                                     R(key, L, DIM_EXTRA + 2), &wi, &sp);
            else
                env_sample(lc, pos, R(key, L, DIM_LIGHT), R(key, L, DIM_LIGHT + 1), &wi, &sp);
        } else if (lc->is_dir) {
            wi = lc->dir;
            sp = pos;
        } else {
            sp = rect_sample(&lc->rect, R2(key, L, DIM_LIGHT));
            wi = normalize(sub(sp, pos));
        }
        const ffo_material* mm = &d->materials[d->material_ids ? d->material_ids[prim] : 0];
        surf_t sf;
        sf.albedo = ld3(mm->base_color);
        sf.fresnel = ld3(mm->fresnel);
        sf.roughness = mm->roughness;
        sf.metallic = mm->metallic;
        sf.ior = mm->ior;
        sf.kind = mm->kind;
        /* ng: the interpolated normal the ray offsets follow (kernel.cu:437);
         * n becomes get_normal's shading normal below */
        v3 ng = n;
        if (d->texcoords && (mm->base_color_tex >= 0 || mm->roughness_tex >= 0 || mm->metallic_tex >= 0 ||
                             mm->metallic_roughness_tex >= 0 || mm->normal_tex >= 0)) {
            /* texcoord = u * uv1 + v * uv2 + (1 - u - v) * uv0 (dTriangle.cu:97) */
            const float* tc = d->texcoords + 6 * (size_t)prim;
            float wuv = (1.f - u) - v;
            float tu = u * tc[2] + v * tc[4] + wuv * tc[0];
            float tv = u * tc[3] + v * tc[5] + wuv * tc[1];
            resolve_textures(mm, d->textures, tu, tv, &sf);
            if (mm->normal_tex >= 0 && d->tangents && d->bitangents) {
                /* the frame interpolated as the normal is (dTriangle.cu:94-96) */
                const float* tg = d->tangents + 9 * (size_t)prim;
                const float* bt = d->bitangents + 9 * (size_t)prim;
                v3 T = normalize(add(add(smul(u, ld3(tg + 3)), smul(v, ld3(tg + 6))), smul((1.f - u) - v, ld3(tg))));
                v3 B = normalize(add(add(smul(u, ld3(bt + 3)), smul(v, ld3(bt + 6))), smul((1.f - u) - v, ld3(bt))));
                const ffo_texture* tx = &d->textures[mm->normal_tex];
                n = normal_from_map(T, B, ng, tex_bilinear(tx->rgb, tx->width, tx->height, tu, tv));
            }
        }
        if (back) {   /* both normals face the ray */
            ng = neg(ng);
            n = neg(n);
        }
        const surf_t* mat = &sf;
        v3 wo = neg(dir);
        memset(&sh, 0, sizeof(sh));
        const int diel = mat->kind == 3;
        if (mat->kind == 0) {
            if (corrected) shade_mix32(lc, mat, pos, n, wo, wi, key, L, &sh);
            else shade_mix(lc, corrected, mat, pos, n, wo, wi, key, L, &sh);
        }
        else if (mat->kind == 1) shade_diffuse(lc, corrected, mat, pos, n, wo, wi, key, L, &sh);
        else if (mat->kind == 2) shade_conductor(lc, corrected, mat, pos, n, wo, wi, key, L, &sh);
        else if (diel) shade_dielectric(lc, mat, pos, n, wo, wi, key, L, back, &sh);
        else shade_coat(lc, mat, pos, n, wo, wi, key, L, &sh);   /* kind 4; ffo_render rejects others */
        /* a dielectric's light may lie on the far side */
        float nee_side = (diel && dot(wi, ng) < 0.f) ? -1.f : 1.f;
        v3 lo = add(pos, muls(ng, nee_side * d->shadow_offset));
        sh.has_nee = light_vis_ray(lc, lo, wi, key, L, DIM_NEE_VIS, &sh.r_nee);
        vis_nee = sh.has_nee && !occluded(d, &sh.r_nee);
        vis_spec = sh.has_spec && !occluded(d, &sh.r_spec);
        vis_diff = sh.has_diff && !occluded(d, &sh.r_diff);
        *n_sh += (uint64_t)(sh.has_nee + sh.has_spec + sh.has_diff);
        /* the reference starts the continuation at the hit point (kernel.cu:643);
         * corrected mode, and every ray leaving a dielectric or an inside
         * vertex, starts off the surface on the side it leaves */
        float side = dot(sh.ext_d, ng) >= 0.f ? 1.f : -1.f;
        o = pos;
        if (corrected || diel || back) o = add(pos, muls(ng, side * d->shadow_offset));
        inside = back != (diel && side < 0.f);
        dir = sh.ext_d;
    }
}

typedef struct {
    const ffo_render_desc* d;
    const light_ctx* lc;
    double* out;
    int row0, row1;
    uint64_t n_ext, n_sh;
} rjob_t;

static void* render_rows(void* arg)
{
    rjob_t* j = (rjob_t*)arg;
    const ffo_render_desc* d = j->d;
    for (int y = j->row0; y < j->row1; ++y)
        for (int x = 0; x < d->width; ++x) {
            double* px = j->out + 3 * ((size_t)y * d->width + x);
            for (int s = 0; s < d->spp; ++s) {
                double c[3];
                path_sample(d, j->lc, x, y, (uint32_t)(d->sample_offset + s), c, &j->n_ext, &j->n_sh);
                px[0] += c[0]; px[1] += c[1]; px[2] += c[2];
            }
        }
    return NULL;
}

int ffo_render(const ffo_render_desc* d, double* out_rgb, uint64_t* stats)
{
    light_ctx lc;
    memset(&lc, 0, sizeof(lc));
    lc.d = d;
    lc.is_env = d->light == -1;
    lc.corrected = d->mode == 1;
    lc.scale = 1.f;
    double *marginal = NULL, *cond = NULL;
    float* pdf = NULL;
    const int n_lights = (d->env_rgb ? 1 : 0) + d->num_area_lights + d->num_dir_lights;
    if (d->light == -2 && (!lc.corrected || n_lights == 0)) return 1;
    if (d->light < -2 || (d->light == -1 && !d->env_rgb)) return 1;
    if (d->light >= d->num_area_lights + d->num_dir_lights) return 1;
    for (int m = 0; m < d->num_materials; ++m)
        if (d->materials[m].kind < 0 || d->materials[m].kind > 4) return 2;   /* a kind this oracle does not restate */
    if (d->env_rgb && (lc.is_env || d->light == -2)) {
        marginal = (double*)malloc(sizeof(double) * d->env_h);
        cond = (double*)malloc(sizeof(double) * (size_t)d->env_w * d->env_h);
        pdf = (float*)malloc(sizeof(float) * (size_t)d->env_w * d->env_h);
        ffo_env_build(d->env_rgb, d->env_w, d->env_h, marginal, cond, pdf, NULL);
        lc.marginal = marginal;
        lc.cond = cond;
        lc.pdf = pdf;
    }
    memset(out_rgb, 0, sizeof(double) * 3 * (size_t)d->width * d->height);
    int nt = d->threads > 0 ? d->threads : 1;
    if (nt > 256) nt = 256;
    pthread_t th[256];
    rjob_t jobs[256];
    int rows = d->height;
    for (int k = 0; k < nt; ++k) {
        jobs[k].d = d;
        jobs[k].lc = &lc;
        jobs[k].out = out_rgb;
        jobs[k].row0 = rows * k / nt;
        jobs[k].row1 = rows * (k + 1) / nt;
        jobs[k].n_ext = jobs[k].n_sh = 0;
        if (pthread_create(&th[k], NULL, render_rows, &jobs[k]) != 0) {
            render_rows(&jobs[k]);
            th[k] = 0;
        }
    }
    uint64_t ne = 0, ns = 0;
    for (int k = 0; k < nt; ++k) {
        if (th[k]) pthread_join(th[k], NULL);
        ne += jobs[k].n_ext;
        ns += jobs[k].n_sh;
    }
    if (stats) { stats[0] = ne; stats[1] = ns; }
    free(marginal);
    free(cond);
    free(pdf);
    return 0;
}

/* ---------------------------------------------------------------------
 * Probe entry points: the restated routines one by one, for the golden
 * vectors of tests/golden/ (made from the reference's own routines).
 * mat8 = base[3], fresnel[3], roughness, metallic; vectors are float[3].
 * ------------------------------------------------------------------- */
static surf_t mat_of(const float* m8)
{
    surf_t m;
    m.albedo = V(m8[0], m8[1], m8[2]);
    m.fresnel = V(m8[3], m8[4], m8[5]);
    m.roughness = m8[6];
    m.metallic = m8[7];
    m.kind = 0;
    return m;
}
static void st3(float* o, v3 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

/* out: diff_f[3], spec_f[3], spec_pdf, BRDF_pdf, BRDF_f[3], fresnel[3], D, G, diff_pdf (17) */
void ffo_probe_material(const float* m8, const float* n3, const float* wi3, const float* wo3, float* out)
{
    surf_t m = mat_of(m8);
    v3 n = ld3(n3), wi = ld3(wi3), wo = ld3(wo3);
    st3(out, diff_f(&m, wi, wo));
    st3(out + 3, spec_f(&m, n, wi, wo));
    out[6] = spec_get_pdf(n, wi, wo, m.roughness);
    out[7] = brdf_pdf(&m, n, wi, wo);
    st3(out + 8, brdf_f(&m, n, wi, wo));
    v3 wh = normalize(add(wo, wi));
    st3(out + 11, fresnel3(m.fresnel, wh, wi));
    out[14] = (float)ggx_ndf(n, wh, m.roughness);
    out[15] = (float)geo_atten(wi, wo, n, m.roughness);
    out[16] = (float)diff_get_pdf();
}
void ffo_probe_diff_sample(const float* n3, float e0, float e1, float* out3) { st3(out3, diff_sample(ld3(n3), e0, e1)); }
void ffo_probe_spec_sample(const float* n3, const float* wo3, float r, float e0, float e1, float* out3)
{
    st3(out3, spec_sample(ld3(n3), ld3(wo3), r, e0, e1));
}
void ffo_probe_concentric_disk(float u0, float u1, float* out2)
{
    v2 u = {u0, u1};
    v2 r = concentric_disk(u);
    out2[0] = r.x;
    out2[1] = r.y;
}
int ffo_probe_upper_bound(const double* list, int size, float val) { return upper_bound_ref(list, size, val); }
void ffo_probe_tex(const float* rgb, int w, int h, float u, float v, float* out3) { st3(out3, tex_bilinear(rgb, w, h, u, v)); }
/* camera: inv16, lens, focal, jitter scale, W, H, px, py, jitter draws (x, y), lens draws (x, y) -> o[3], d[3] */
void ffo_probe_camera(const float* inv16, float lens, float focal, float jitter, int W, int H, int px, int py,
                      const float* jit2, const float* lens2, float* out6)
{
    ffo_render_desc d;
    memset(&d, 0, sizeof(d));
    for (int k = 0; k < 16; ++k) d.cam_inv[k] = inv16[k];
    d.cam_lens_radius = lens;
    d.cam_focal = focal;
    d.cam_jitter = jitter;
    d.width = W;
    d.height = H;
    v2 j = {jit2[0], jit2[1]}, l = {lens2[0], lens2[1]};
    v3 o, dir;
    camera_ray(&d, px, py, j, l, &o, &dir);
    st3(out6, o);
    st3(out6 + 3, dir);
}
/* environment: sample (ex, ey) from tables, L and pdf of a direction */
void ffo_probe_env(const float* rgb, int w, int h, const double* marginal, const double* cond, const float* pdf,
                   const float* pos3, float ex, float ey, const float* q3, float* out)
{
    ffo_render_desc d;
    memset(&d, 0, sizeof(d));
    d.env_rgb = rgb;
    d.env_w = w;
    d.env_h = h;
    light_ctx lc;
    memset(&lc, 0, sizeof(lc));
    lc.d = &d;
    lc.is_env = 1;
    lc.marginal = marginal;
    lc.cond = cond;
    lc.pdf = pdf;
    v3 wi, sp;
    env_sample(&lc, ld3(pos3), ex, ey, &wi, &sp);
    st3(out, wi);
    st3(out + 3, sp);
    st3(out + 6, env_L(&d, ld3(q3)));
    out[9] = env_pdf(&lc, ld3(q3));
}
/* area light: sample point from draws (x, y), L(wi), pdf with redraw (x, y), rect hit */
void ffo_probe_area(const ffo_area_light* L, const float* pos3, const float* u2, const float* wi3, const float* u2pdf,
                    const float* ray8, float* out)
{
    rect_t r = make_rect(L);
    v2 u = {u2[0], u2[1]}, up = {u2pdf[0], u2pdf[1]};
    v3 sp = rect_sample(&r, u);
    st3(out, sp);
    st3(out + 3, normalize(sub(sp, ld3(pos3))));
    st3(out + 6, rect_L(&r, ld3(wi3)));
    out[9] = rect_pdf(&r, ld3(pos3), up);
    v3 o = V(ray8[0], ray8[1], ray8[2]), dd = V(ray8[4], ray8[5], ray8[6]);
    out[10] = (float)rect_hit(&r, o, dd);
}

/* Probe of the material texture reads: isect11 = texcoord[2], normal[3],
 * tangent[3], bitangent[3] (as dTriangle::hit leaves them); out8 = albedo[3],
 * roughness, metallic, normal[3]. */
void ffo_probe_surface(const ffo_material* mm, const ffo_texture* textures, const float* isect11, float* out8)
{
    surf_t sf;
    sf.albedo = ld3(mm->base_color);
    sf.fresnel = ld3(mm->fresnel);
    sf.roughness = mm->roughness;
    sf.metallic = mm->metallic;
    sf.kind = mm->kind;
    resolve_textures(mm, textures, isect11[0], isect11[1], &sf);
    v3 N = ld3(isect11 + 2);
    if (mm->normal_tex >= 0) {
        const ffo_texture* tx = &textures[mm->normal_tex];
        N = normal_from_map(ld3(isect11 + 5), ld3(isect11 + 8), N,
                            tex_bilinear(tx->rgb, tx->width, tx->height, isect11[0], isect11[1]));
    }
    st3(out8, sf.albedo);
    out8[3] = sf.roughness;
    out8[4] = sf.metallic;
    st3(out8 + 5, N);
}

/* Dielectric and coat probes (the restated lobes one call at a time, for
 * the known-answer tests of tests/test_oracle_materials_cpu.py).
 * mat5 = base colour (tint / albedo) [3], roughness, ior. */
static surf_t mat5_of(const float* m5)
{
    surf_t m;
    memset(&m, 0, sizeof(m));
    m.albedo = ld3(m5);
    m.fresnel = V(0.04f, 0.04f, 0.04f);
    m.roughness = m5[3];
    m.ior = m5[4];
    return m;
}
void ffo_probe_dielectric(const float* mat5, int back, const float* n3, const float* wo3, const float* wi3, float* out4)
{
    surf_t m = mat5_of(mat5);
    diel_t d = diel_of(&m, back);
    v3 f;
    float pdf;
    diel_eval(&d, ld3(n3), ld3(wo3), ld3(wi3), &f, &pdf);
    st3(out4, f);
    out4[3] = pdf;
}
int ffo_probe_dielectric_sample(const float* mat5, int back, const float* n3, const float* wo3, float e0, float e1,
                                float e2, float* wi3)
{
    surf_t m = mat5_of(mat5);
    diel_t d = diel_of(&m, back);
    v3 wi = V(0, 0, 0);
    int ok = diel_sample(&d, ld3(n3), ld3(wo3), e0, e1, e2, &wi);
    st3(wi3, wi);
    return ok;
}
float ffo_probe_fresnel_dielectric(float c, float n) { return fresnel_dielectric(c, n); }
void ffo_probe_coat(const float* mat5, const float* n3, const float* wi3, const float* wo3, float* out4)
{
    surf_t m = mat5_of(mat5);
    float eta = m.ior > 0.f ? m.ior : 1.5f;
    float r0 = ((eta - 1.f) / (eta + 1.f)) * ((eta - 1.f) / (eta + 1.f));
    v3 n = ld3(n3), wi = ld3(wi3), wo = ld3(wo3);
    st3(out4, coat_f(&m, n, wi, wo, r0));
    float c = hmax(0.f, dot(n, wi));
    out4[3] = 0.5f * spec_get_pdf32(n, wi, wo, m.roughness) + 0.5f * c * INV_PI_F;
}
