// ffref_harness.cpp — C entry points over the reference's own routines,
// compiled for the host (see ffref_compat.h).  TEST INFRASTRUCTURE ONLY:
// oracle/_ref/libffref.so pins the oracle's restatement (golden vectors in
// tests/golden/) and serves as the timed CPU baseline of the trace workload.
//
// Everything that calls a reference routine below calls the unmodified code
// from CUDA-RayTracer/ (dTriangle.cu, BVH.cpp, dRandom.cu, dMaterial.cu,
// dEnvironmentLight.cu, dAreaLight.cu, Rectangle.cuh, dCamera.cu, Helpers.cu).
// The only logic restated here is the environment-table build of
// kernel.cu:65-149, which cannot be compiled for the host (kernel.cu pulls in
// GL headers and the removed surface-reference API).
#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <thread>

#include "BVH.h"
#include "Helpers.cuh"
#include "Isect.cuh"
#include "Rectangle.cuh"
#include "dAreaLight.cuh"
#include "dCamera.cuh"
#include "dEnvironmentLight.cuh"
#include "dFilm.cuh"
#include "dMaterial.cuh"
#include "dMath.cuh"
#include "dRandom.cuh"
#include "dTriangle.cuh"

thread_local uint3 threadIdx = {0, 0, 0};
thread_local uint3 blockIdx = {0, 0, 0};
thread_local dim3 blockDim = dim3(1, 1, 1);

// ------------------------------------------------------------ clock control
static thread_local const uint32_t* g_seq = nullptr;
static thread_local int g_seq_n = 0;
static thread_local int g_seq_i = 0;

// Without a sequence (the timed renders), clock() advances a per-thread
// counter so every random() call draws a new value, as a running clock does.
static thread_local uint32_t g_free_clock = 0;

long ffref_clock(void)
{
    if (g_seq && g_seq_i < g_seq_n) return (long)g_seq[g_seq_i++];
    ++g_seq_i;
    if (!g_seq) return (long)(g_free_clock += 7919u);
    return 0;
}

// Every visibility query of the reference goes through intersect_shadows
// (dTriangle.cu:215-259), called from the lights' visible().  The library is
// linked with --wrap for that symbol so the renders can count the rays.
static thread_local uint64_t g_shadow_calls = 0;
extern "C" bool __real__Z17intersect_shadowsPK13LinearBVHNodePK9dTriangleRK4dRayRf(const LinearBVHNode*,
                                                                                  const dTriangle*, const dRay&,
                                                                                  float&);
extern "C" bool __wrap__Z17intersect_shadowsPK13LinearBVHNodePK9dTriangleRK4dRayRf(const LinearBVHNode* n,
                                                                                  const dTriangle* t, const dRay& r,
                                                                                  float& tmin)
{
    ++g_shadow_calls;
    return __real__Z17intersect_shadowsPK13LinearBVHNodePK9dTriangleRK4dRayRf(n, t, r, tmin);
}

// ---------------------------------------------------- texture emulation
struct HostTex {
    int w = 0, h = 0;
    std::vector<float> rgba;  // 4 floats per texel
};
static std::mutex g_tex_mu;
static std::map<unsigned long long, HostTex> g_tex;
static unsigned long long g_next_tex = 1;

// Bilinear fetch with normalised coordinates, wrap addressing and 8-bit
// fractional weights, as the CUDA Programming Guide describes linear
// texture filtering (x_B = x*W - 0.5, alpha = frac(x_B) in 9-bit fixed point
// with 8 fractional bits).
void ffref_tex_fetch(unsigned long long obj, float u, float v, float out[4])
{
    const HostTex* t;
    {
        std::lock_guard<std::mutex> lk(g_tex_mu);
        auto it = g_tex.find(obj);
        if (it == g_tex.end()) {
            out[0] = out[1] = out[2] = out[3] = 0.f;
            return;
        }
        t = &it->second;
    }
    float xb = u * (float)t->w - 0.5f;
    float yb = v * (float)t->h - 0.5f;
    float fx = floorf(xb), fy = floorf(yb);
    float ax = xb - fx, ay = yb - fy;
    ax = floorf(ax * 256.f + 0.5f) / 256.f;
    ay = floorf(ay * 256.f + 0.5f) / 256.f;
    long ix = (long)fx, iy = (long)fy;
    auto wrap = [](long i, int n) { long r = i % n; return (int)(r < 0 ? r + n : r); };
    int x0 = wrap(ix, t->w), x1 = wrap(ix + 1, t->w), y0 = wrap(iy, t->h), y1 = wrap(iy + 1, t->h);
    for (int c = 0; c < 4; ++c) {
        float t00 = t->rgba[4 * (y0 * t->w + x0) + c], t10 = t->rgba[4 * (y0 * t->w + x1) + c];
        float t01 = t->rgba[4 * (y1 * t->w + x0) + c], t11 = t->rgba[4 * (y1 * t->w + x1) + c];
        out[c] = (1.f - ax) * (1.f - ay) * t00 + ax * (1.f - ay) * t10 + (1.f - ax) * ay * t01 + ax * ay * t11;
    }
}

void ffref_surf_read_float(unsigned long long obj, int x_bytes, int y, float* out)
{
    std::lock_guard<std::mutex> lk(g_tex_mu);
    auto it = g_tex.find(obj);
    if (it == g_tex.end()) {
        *out = 0.f;
        return;
    }
    const HostTex& t = it->second;
    int x = x_bytes / 4;
    if (x < 0 || y < 0 || x >= t.w || y >= t.h) {
        *out = 0.f;
        return;
    }
    *out = t.rgba[4 * (y * t.w + x)];
}

extern "C" {
void ffref_env_free(void* h);
void ffref_area_free(void* h);
void* ffref_env_create(const float* rgb, int w, int h);
void* ffref_area_create(const float* rect12, float radiance, const float* emissive3);

// ------------------------------------------------------------------ misc
void ffref_set_clock(const uint32_t* seq, int n)
{
    g_seq = seq;
    g_seq_n = n;
    g_seq_i = 0;
}
int ffref_clock_used(void) { return g_seq_i; }

unsigned long long ffref_tex_create(const float* rgb, int w, int h, int channels)
{
    HostTex t;
    t.w = w;
    t.h = h;
    t.rgba.assign((size_t)4 * w * h, 0.f);
    for (int i = 0; i < w * h; ++i)
        for (int c = 0; c < channels && c < 4; ++c) t.rgba[4 * i + c] = rgb[channels * i + c];
    std::lock_guard<std::mutex> lk(g_tex_mu);
    unsigned long long id = g_next_tex++;
    g_tex[id] = std::move(t);
    return id;
}

void ffref_tex_sample(unsigned long long obj, float u, float v, float* out4)
{
    float4 s = tex2DLod<float4>(obj, u, v, 0);
    out4[0] = s.x;
    out4[1] = s.y;
    out4[2] = s.z;
    out4[3] = s.w;
}

// -------------------------------------------------------------- triangles
static dTriangle make_tri(const float* p)
{
    dVertex a{}, b{}, c{};
    a.position = make_float3(p[0], p[1], p[2]);
    b.position = make_float3(p[3], p[4], p[5]);
    c.position = make_float3(p[6], p[7], p[8]);
    return dTriangle(a, b, c);
}

int ffref_intersect(const float* tri9, const float* ray8, float* tuv)
{
    dTriangle t = make_tri(tri9);
    dRay r(make_float3(ray8[0], ray8[1], ray8[2]), make_float3(ray8[4], ray8[5], ray8[6]));
    float u = 0, v = 0, tt = 0;
    int ok = t.intersect(r, u, v, tt) ? 1 : 0;
    tuv[0] = tt;
    tuv[1] = u;
    tuv[2] = v;
    return ok;
}

int ffref_shadow_hit(const float* tri9, const float* ray8, float* t_out)
{
    dTriangle t = make_tri(tri9);
    dRay r(make_float3(ray8[0], ray8[1], ray8[2]), make_float3(ray8[4], ray8[5], ray8[6]));
    float tt = 0;
    int ok = t.shadow_hit(r, tt) ? 1 : 0;
    *t_out = tt;
    return ok;
}

// ------------------------------------------------------------------- BVH
struct RefBVH {
    std::vector<dTriangle> tris;       // reordered as d_reorder_primitives does
    std::vector<int> ordered;          // orderedPrims: position -> original index
    LinearBVHNode* nodes = nullptr;
    int num_nodes = 0;
    dMaterial mat;
};

// BVHAccel(SAH, 8) over the triangles' bounds, as dScene::init_BVH
// (dScene.cpp:324-379) sets it up, then the reorder of kernel.cu:184-191.
void* ffref_bvh_build(const float* tris9, int n, double* build_ms)
{
    auto t0 = std::chrono::steady_clock::now();
    RefBVH* b = new RefBVH();
    std::vector<dTriangle> src;
    src.reserve(n);
    std::vector<BVHPrimitiveInfo> info;
    info.reserve(n);
    for (int i = 0; i < n; ++i) {
        src.push_back(make_tri(tris9 + 9 * i));
        src.back().material = &b->mat;
        const float* p = tris9 + 9 * i;
        Bounds3f bb = Union(Bounds3f(make_float3(p[0], p[1], p[2]), make_float3(p[3], p[4], p[5])),
                            make_float3(p[6], p[7], p[8]));
        info.emplace_back((size_t)i, bb);
    }
    BVHAccel accel(info, SplitMethod::SAH, 8);
    b->ordered = accel.get_ordered_prims();
    b->num_nodes = accel.get_nmb_nodes();
    b->nodes = accel.get_nodes();
    b->tris.resize(n);
    for (int i = 0; i < n; ++i) b->tris[i] = src[b->ordered[i]];
    auto t1 = std::chrono::steady_clock::now();
    if (build_ms) *build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return b;
}

int ffref_bvh_num_nodes(void* h) { return ((RefBVH*)h)->num_nodes; }

// The host build's arrays, for uploading the same BVH to the reference's
// own GPU traversal (oracle/_ref/libffrefcuda.so): nodes, reordered
// triangles, the position -> original index map, and the struct sizes.
void ffref_bvh_data(void* h, const void** nodes, const void** tris, const int** ordered, int* num_tris)
{
    RefBVH* b = (RefBVH*)h;
    *nodes = b->nodes;
    *tris = b->tris.data();
    *ordered = b->ordered.data();
    *num_tris = (int)b->tris.size();
}

void ffref_sizes(int* node_bytes, int* tri_bytes, int* isect_bytes)
{
    *node_bytes = (int)sizeof(LinearBVHNode);
    *tri_bytes = (int)sizeof(dTriangle);
    *isect_bytes = (int)sizeof(Isect);
}

void ffref_bvh_free(void* h) { delete (RefBVH*)h; }

// intersect() / intersect_shadows() (dTriangle.cu:140-259) per ray over
// nthreads threads.  hits: t (float), prim (int32, original index), 8 bytes
// per ray.  Closest-hit reports the reference's own choice among equal t
// (its traversal order).  Any-hit uses tmax = ray[7].
void ffref_bvh_trace(void* h, const float* rays, long n, void* hits, int any, int nthreads)
{
    RefBVH* b = (RefBVH*)h;
    if (nthreads < 1) nthreads = 1;
    std::atomic<long> next{0};
    const long chunk = 1024;
    auto work = [&]() {
        for (;;) {
            long s = next.fetch_add(chunk);
            if (s >= n) break;
            long e = std::min(n, s + chunk);
            for (long i = s; i < e; ++i) {
                const float* r = rays + 8 * i;
                dRay ray(make_float3(r[0], r[1], r[2]), make_float3(r[4], r[5], r[6]));
                float* ho = (float*)hits + 2 * i;
                int32_t prim = -1;
                float t = r[7];
                if (any) {
                    float tmax = r[7];
                    if (intersect_shadows(b->nodes, b->tris.data(), ray, tmax)) prim = 0;
                } else {
                    Isect is;
                    intersect(b->nodes, b->tris.data(), ray, is);
                    if (is.wasFound) {
                        prim = b->ordered[is.triangle_id];
                        t = is.distance;
                    }
                }
                ho[0] = t;
                std::memcpy(ho + 1, &prim, 4);
            }
        }
    };
    std::vector<std::thread> th;
    for (int k = 1; k < nthreads; ++k) th.emplace_back(work);
    work();
    for (auto& x : th) x.join();
}

// --------------------------------------------------------------- sampler
uint32_t ffref_wang_hash(uint32_t s) { return wang_hash(s); }

// random() (renamed ffref_random by the shim) with the clock sequence set
// by ffref_set_clock.
float ffref_rand_draw(void) { return random(); }

void ffref_uniform_sample_square(float* out2)
{
    float2 p = UniformSampleSquare();
    out2[0] = p.x;
    out2[1] = p.y;
}
void ffref_concentric_sample_disk(const float* u2, float* out2)
{
    float2 p = ConcentricSampleDisk(make_float2(u2[0], u2[1]));
    out2[0] = p.x;
    out2[1] = p.y;
}
void ffref_concentric_sample_disk_drawn(float* out2)
{
    float2 p = ConcentricSampleDisk();
    out2[0] = p.x;
    out2[1] = p.y;
}
void ffref_uniform_sample_hemisphere(const float* u2, float* out3)
{
    float3 p = UniformSampleHemisphere(make_float2(u2[0], u2[1]));
    out3[0] = p.x;
    out3[1] = p.y;
    out3[2] = p.z;
}
void ffref_uniform_sample_sphere(const float* u2, float* out3)
{
    float3 p = UniformSampleSphere(make_float3(u2[0], u2[1], 0.f));
    out3[0] = p.x;
    out3[1] = p.y;
    out3[2] = p.z;
}

// -------------------------------------------------------------- materials
// Material record passed from Python: base[3], fresnel[3], roughness,
// metallic (8 floats); isect: position[3], normal[3] (6 floats).
static void fill(dMaterial& m, Isect& is, const float* mat8, const float* isect6)
{
    m.baseColorFactor = make_float3(mat8[0], mat8[1], mat8[2]);
    m.fresnel = make_float3(mat8[3], mat8[4], mat8[5]);
    m.roughnessFactor = mat8[6];
    m.metallicFactor = mat8[7];
    is.position = make_float3(isect6[0], isect6[1], isect6[2]);
    is.normal = make_float3(isect6[3], isect6[4], isect6[5]);
    is.material = &m;
    is.wasFound = true;
}

// out: diff_f[3], spec_f[3], spec_pdf, BRDF_pdf, BRDF_f[3], fresnel[3],
// ggxtr_ndf (as float), geo_atten (as float), diff_get_pdf  (19 floats)
void ffref_material_eval(const float* mat8, const float* isect6, const float* wi3, const float* wo3, float* out)
{
    dMaterial m;
    Isect is;
    fill(m, is, mat8, isect6);
    float3 wi = make_float3(wi3[0], wi3[1], wi3[2]);
    float3 wo = make_float3(wo3[0], wo3[1], wo3[2]);
    float3 df = diff_f(is, wi, wo);
    float3 sf = spec_f(is, wi, wo);
    float sp = spec_get_pdf(get_normal(is), wi, wo, get_roughness(is));
    float bp = BRDF_pdf(is, wi, wo);
    float3 bf = BRDF_f(is, wi, wo);
    float3 wh = normalize(wo + wi);
    float3 F = fresnel(make_float3(mat8[3], mat8[4], mat8[5]), wh, wi);
    double D = ggxtr_ndf(get_normal(is), wh, get_roughness(is));
    double G = geo_atten(wi, wo, get_normal(is), get_roughness(is));
    float vals[19] = {df.x, df.y, df.z, sf.x, sf.y, sf.z, sp, bp, bf.x, bf.y, bf.z, F.x, F.y, F.z,
                      (float)D, (float)G, (float)diff_get_pdf(), 0.f, 0.f};
    std::memcpy(out, vals, sizeof(vals));
}

void ffref_diff_sample(const float* mat8, const float* isect6, float* out3)
{
    dMaterial m;
    Isect is;
    fill(m, is, mat8, isect6);
    float3 w = diff_sample(is);
    out3[0] = w.x;
    out3[1] = w.y;
    out3[2] = w.z;
}

void ffref_spec_sample(const float* mat8, const float* isect6, const float* wo3, float* out3)
{
    dMaterial m;
    Isect is;
    fill(m, is, mat8, isect6);
    float3 w = spec_sample(is, make_float3(wo3[0], wo3[1], wo3[2]));
    out3[0] = w.x;
    out3[1] = w.y;
    out3[2] = w.z;
}

double ffref_power_heuristic(int nf, double f, int ng, double g) { return power_heuristic(nf, f, ng, g); }

// get_albedo / get_roughness / get_metallic / get_normal (dMaterial.cu:10-88)
// with material textures.  mat8: base colour[3], fresnel[3], roughness and
// metallic factors; tex5: texture objects (ffref_tex_create) for the base
// colour, roughness, metallic, metallic-roughness and normal slots, -1 none;
// isect11: texcoord[2], normal[3], tangent[3], bitangent[3] (as dTriangle::hit
// leaves them).  out8: albedo[3], roughness, metallic, normal[3].
void ffref_surface(const float* mat8, const int* tex5, const float* isect11, float* out8)
{
    dMaterial m;
    Isect is;
    fill(m, is, mat8, isect11);   // position / normal slots overwritten below
    m.baseColorTexture = tex5[0];
    m.roughnessTexture = tex5[1];
    m.metallicTexture = tex5[2];
    m.metallicRoughnessTexture = tex5[3];
    m.normalTexture = tex5[4];
    is.texcoord = make_float2(isect11[0], isect11[1]);
    is.normal = make_float3(isect11[2], isect11[3], isect11[4]);
    is.tangent = make_float3(isect11[5], isect11[6], isect11[7]);
    is.bitangent = make_float3(isect11[8], isect11[9], isect11[10]);
    const float3 a = get_albedo(is);
    const float r = get_roughness(is);
    const float mt = get_metallic(is);
    const float3 n = get_normal(is);
    const float vals[8] = {a.x, a.y, a.z, r, mt, n.x, n.y, n.z};
    std::memcpy(out8, vals, sizeof(vals));
}

// ------------------------------------------------------------------ camera
// gen_ray (dCamera.cu:10-36) for pixel (px, py): cam = inv_view_proj[16]
// (Matrix4x4 m[i][j] at 4*i+j), lens_radius, f.  out = o[3], d[3].
void ffref_gen_ray(const float* inv16, float lens_radius, float focal, int hres, int vres, float px, float py,
                   float* out6)
{
    dFilm film;
    film.hres = hres;
    film.vres = vres;
    dCamera cam;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) cam.inv_view_proj_mat.m[i][j] = inv16[4 * i + j];
    cam.lens_radius = lens_radius;
    cam.f = focal;
    dRay r = cam.gen_ray(&film, make_float2(px, py));
    out6[0] = r.o.x;
    out6[1] = r.o.y;
    out6[2] = r.o.z;
    out6[3] = r.d.x;
    out6[4] = r.d.y;
    out6[5] = r.d.z;
}

// ---------------------------------------------------------------- lights
// Environment tables: the serial loops of kernel.cu:65-149 (the one piece
// restated here), over the emulated texture.  marginal_y[h], conds[h*w],
// pdf[h*w] (already scaled by w*h/(2*pi^2)), *denom.
struct RefEnv {
    unsigned long long tex = 0, surf = 0;
    int w = 0, h = 0;
    std::vector<double> marginal_y, marginal_p;
    std::vector<std::vector<double>> conds;
    std::vector<double*> cond_ptrs;
    double denom = 0;
    dEnvironmentLight* light = nullptr;
};

void* ffref_env_create(const float* rgb, int w, int h)
{
    RefEnv* e = new RefEnv();
    e->w = w;
    e->h = h;
    e->tex = ffref_tex_create(rgb, w, h, 3);
    // g_compute_pdf_denom (kernel.cu:65-84)
    double denom = 0.0;
    for (int j = 0; j < h; j++) {
        float v = (float)j / (float)h;
        double sin_theta = sin(M_PI * v);
        for (int i = 0; i < w; i++) {
            float u = (float)i / (float)w;
            float4 s = tex2DLod<float4>(e->tex, u, v, 0);
            double lum = luminance(make_float3(s.x, s.y, s.z));
            denom += lum * sin_theta;
        }
    }
    e->denom = denom;
    // g_compute_marginal_dist (kernel.cu:86-108)
    e->marginal_y.assign(h, 0.0);
    e->marginal_p.assign(h, 0.0);
    for (int j = 0; j < h; j++) {
        float v = (float)j / (float)h;
        double sin_theta = sin(M_PI * v) / denom;
        e->marginal_p[j] = 0.f;
        for (int i = 0; i < w; i++) {
            float u = (float)i / (float)w;
            float4 s = tex2DLod<float4>(e->tex, u, v, 0);
            double lum = luminance(make_float3(s.x, s.y, s.z));
            e->marginal_p[j] += lum * sin_theta;
        }
        if (j != 0) e->marginal_y[j] = e->marginal_p[j] + e->marginal_y[j - 1];
        else e->marginal_y[j] = e->marginal_p[j];
    }
    // g_compute_conditional_dist (kernel.cu:110-128)
    e->conds.assign(h, std::vector<double>(w, 0.0));
    for (int y = 0; y < h; y++) {
        float v = (float)y / (float)h;
        double sin_theta = sin(M_PI * v);
        double val = sin_theta / (denom * e->marginal_p[y]);
        for (int x = 0; x < w; x++) {
            float u = (float)x / (float)w;
            float4 s = tex2DLod<float4>(e->tex, u, v, 0);
            double lum = luminance(make_float3(s.x, s.y, s.z));
            e->conds[y][x] = lum * val;
            if (x != 0) e->conds[y][x] += e->conds[y][x - 1];
        }
    }
    for (auto& row : e->conds) e->cond_ptrs.push_back(row.data());
    // g_write_pdf_texture (kernel.cu:130-149)
    std::vector<float> pdf((size_t)w * h);
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
            float u = (float)x / (float)w;
            float v = (float)y / (float)h;
            double sin_theta = sin(M_PI * v);
            float4 s = tex2DLod<float4>(e->tex, u, v, 0);
            double lum = luminance(make_float3(s.x, s.y, s.z));
            float p = (lum * sin_theta) / denom;
            p *= (w * h) / (2.f * M_PI * M_PI);
            pdf[(size_t)y * w + x] = p;
        }
    }
    e->surf = ffref_tex_create(pdf.data(), w, h, 1);
    e->light = new dEnvironmentLight(e->tex, e->surf, e->marginal_y.data(), e->cond_ptrs.data(), w, h);
    return e;
}

void ffref_env_tables(void* h, double* marginal, double* conds, float* pdf, double* denom)
{
    RefEnv* e = (RefEnv*)h;
    if (marginal) std::memcpy(marginal, e->marginal_y.data(), sizeof(double) * e->h);
    if (conds)
        for (int y = 0; y < e->h; ++y) std::memcpy(conds + (size_t)y * e->w, e->conds[y].data(), sizeof(double) * e->w);
    if (pdf) {
        float v[4];
        for (int y = 0; y < e->h; ++y)
            for (int x = 0; x < e->w; ++x) {
                ffref_surf_read_float(e->surf, 4 * x, y, v);
                pdf[(size_t)y * e->w + x] = v[0];
            }
    }
    if (denom) *denom = e->denom;
}

// get_direction (2 draws from the clock sequence), L, get_pdf(isect, wi)
void ffref_env_sample(void* h, const float* pos3, float* wi3, float* sp3)
{
    RefEnv* e = (RefEnv*)h;
    Isect is;
    is.position = make_float3(pos3[0], pos3[1], pos3[2]);
    float3 wi, sp;
    e->light->get_direction(is, wi, sp);
    wi3[0] = wi.x;
    wi3[1] = wi.y;
    wi3[2] = wi.z;
    sp3[0] = sp.x;
    sp3[1] = sp.y;
    sp3[2] = sp.z;
}

void ffref_env_eval(void* h, const float* wi3, float* L3, float* pdf)
{
    RefEnv* e = (RefEnv*)h;
    Isect is;
    float3 wi = make_float3(wi3[0], wi3[1], wi3[2]);
    float3 L = e->light->L(is, wi, make_float3(0.f));
    L3[0] = L.x;
    L3[1] = L.y;
    L3[2] = L.z;
    *pdf = e->light->get_pdf(is, wi);
}

int ffref_upper_bound(const double* list, int size, float val) { return upper_bound((double*)list, size, val); }

void ffref_env_free(void* h)
{
    RefEnv* e = (RefEnv*)h;
    delete e->light;
    delete e;
}

// Area light: _Rectangle + dAreaLight.  rect = p0[3], a[3], b[3], n[3];
// material radiance and emissive colour.
struct RefArea {
    _Rectangle* rect = nullptr;
    dAreaLight* light = nullptr;
    dMaterial mat;
};

void* ffref_area_create(const float* rect12, float radiance, const float* emissive3)
{
    RefArea* a = new RefArea();
    a->rect = new _Rectangle(make_float3(rect12[0], rect12[1], rect12[2]), make_float3(rect12[3], rect12[4], rect12[5]),
                             make_float3(rect12[6], rect12[7], rect12[8]), make_float3(rect12[9], rect12[10], rect12[11]));
    a->light = new dAreaLight();
    a->light->set_object(a->rect);
    a->mat.radiance = radiance;
    a->mat.emissiveColorFactor = make_float3(emissive3[0], emissive3[1], emissive3[2]);
    a->light->material = &a->mat;
    return a;
}

// get_direction: sample() (2 draws).  L(wi).  get_pdf(isect, wi) (2 draws).
void ffref_area_sample(void* h, const float* pos3, float* wi3, float* sp3)
{
    RefArea* a = (RefArea*)h;
    Isect is;
    is.position = make_float3(pos3[0], pos3[1], pos3[2]);
    float3 wi, sp;
    a->light->get_direction(is, wi, sp);
    wi3[0] = wi.x;
    wi3[1] = wi.y;
    wi3[2] = wi.z;
    sp3[0] = sp.x;
    sp3[1] = sp.y;
    sp3[2] = sp.z;
}

void ffref_area_eval(void* h, const float* pos3, const float* wi3, const float* sp3, float* L3, float* pdf)
{
    RefArea* a = (RefArea*)h;
    Isect is;
    is.position = make_float3(pos3[0], pos3[1], pos3[2]);
    float3 wi = make_float3(wi3[0], wi3[1], wi3[2]);
    float3 L = a->light->L(is, wi, make_float3(sp3[0], sp3[1], sp3[2]));
    L3[0] = L.x;
    L3[1] = L.y;
    L3[2] = L.z;
    *pdf = a->light->get_pdf(is, wi);
}

// _Rectangle::hit(ray) (Rectangle.cuh:74-97)
int ffref_area_hit(void* h, const float* ray8)
{
    RefArea* a = (RefArea*)h;
    dRay r(make_float3(ray8[0], ray8[1], ray8[2]), make_float3(ray8[4], ray8[5], ray8[6]));
    return a->rect->hit(r) ? 1 : 0;
}

// ------------------------------------------------------------------ render
// The reference's path tracer on the host: dCamera::gen_ray, intersect()
// over its SAH BVH, the lights' get_direction / L / visible, and BRDF_L /
// BRDF_f / BRDF_pdf of the mix material (with their inline visibility
// traversals), driven by a restatement of the per-path logic of wf_logic /
// wf_generate / wf_mat_mix / wf_extend / wf_shadow (kernel.cu:298-651): one
// path per pixel sample, one bounce per iteration.  random() draws from the
// free-running per-thread clock.  Pixels rendered: every `pixel_stride`-th
// pixel (all of them for 1).  out_rgb (w*h*3 floats, may be NULL) receives
// the radiance sums; stats[0..2] = extension rays, visibility rays, samples.
struct RenderDesc {
    const float* tris;           // T x 9
    const float* normals;        // T x 9 vertex normals
    const uint32_t* material_ids;
    int num_tris;
    const float* mats;           // M x 8: base[3], fresnel[3], roughness, metallic
    int num_mats;
    const float* env_rgb;        // env_h x env_w x 3 or NULL
    int env_w, env_h;
    const float* rect;           // 12 floats + radiance + emissive[3], or NULL
    const float* cam_inv;        // 16
    float lens_radius, focal;
    int width, height, spp, max_depth, rr_depth, light_env, threads, pixel_stride;
};

void ffref_render(const RenderDesc* d, float* out_rgb, uint64_t* stats, double* ms)
{
    auto t0 = std::chrono::steady_clock::now();
    double bms = 0;
    RefBVH* bvh = (RefBVH*)ffref_bvh_build(d->tris, d->num_tris, &bms);
    std::vector<dMaterial> mats(d->num_mats);
    for (int m = 0; m < d->num_mats; ++m) {
        const float* p = d->mats + 8 * m;
        mats[m].baseColorFactor = make_float3(p[0], p[1], p[2]);
        mats[m].fresnel = make_float3(p[3], p[4], p[5]);
        mats[m].roughnessFactor = p[6];
        mats[m].metallicFactor = p[7];
    }
    // vertex normals and materials into the reordered triangles
    for (int i = 0; i < d->num_tris; ++i) {
        int orig = bvh->ordered[i];
        const float* n = d->normals + 9 * (size_t)orig;
        bvh->tris[i].v0.normal = make_float3(n[0], n[1], n[2]);
        bvh->tris[i].v1.normal = make_float3(n[3], n[4], n[5]);
        bvh->tris[i].v2.normal = make_float3(n[6], n[7], n[8]);
        bvh->tris[i].material = &mats[d->material_ids ? d->material_ids[orig] : 0];
    }
    RefEnv* env = nullptr;
    RefArea* area = nullptr;
    dLight* lights[2] = {nullptr, nullptr};
    int light_id = 0;
    if (d->light_env) {
        env = (RefEnv*)ffref_env_create(d->env_rgb, d->env_w, d->env_h);
        lights[0] = env->light;
    } else {
        area = (RefArea*)ffref_area_create(d->rect, d->rect[12], d->rect + 13);
        lights[0] = area->light;
    }
    dFilm film;
    film.hres = d->width;
    film.vres = d->height;
    const int stride = d->pixel_stride > 0 ? d->pixel_stride : 1;
    const long npix = ((long)d->width * d->height + stride - 1) / stride;
    std::atomic<long> next{0};
    std::atomic<uint64_t> n_ext{0}, n_sh{0}, n_samp{0};
    auto work = [&](int tid) {
        g_free_clock = 0x9e3779b9u * (uint32_t)(tid + 1);
        dCamera cam;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) cam.inv_view_proj_mat.m[i][j] = d->cam_inv[4 * i + j];
        cam.lens_radius = d->lens_radius;
        cam.f = d->focal;
        uint64_t ext = 0, samples = 0;
        g_shadow_calls = 0;
        for (;;) {
            long k = next.fetch_add(64);
            if (k >= npix) break;
            long kend = std::min(npix, k + 64);
            for (long q = k; q < kend; ++q) {
                long pix = q * stride;
                int x = (int)(pix % d->width), y = (int)(pix / d->width);
                float3 acc = make_float3(0.f);
                for (int s = 0; s < d->spp; ++s) {
                    // wf_generate
                    dRay ray = cam.gen_ray(&film, make_float2((float)x, (float)y));
                    float3 beta = make_float3(1.f);
                    uint32_t L = 0;
                    float3 light_brdf = make_float3(0.f), ext_brdf = make_float3(0.f);
                    float ext_pdf = 0.f, ext_cos = 0.f;
                    bool light_visible = false;
                    for (;;) {
                        // wf_extend
                        Isect is;
                        intersect(bvh->nodes, bvh->tris.data(), ray, is);
                        ++ext;
                        ++L;
                        // wf_logic
                        bool terminate = (L > (uint32_t)d->max_depth) || !is.wasFound;
                        if (!is.wasFound && L == 1 && env) {
                            float3 sp;
                            acc += beta * env->light->L(is, ray.d, sp);
                        }
                        if (L > 1) {
                            if (light_visible) acc += light_brdf * beta;
                            if (ext_brdf == make_float3(0, 0, 0) || ext_pdf == 0.f) {
                                terminate = true;
                            } else {
                                beta *= ext_brdf * ext_cos / ext_pdf;
                                if (L > (uint32_t)d->rr_depth) {
                                    float q_rr = fmaxf((float).05, 1 - beta.y);
                                    if (random() < q_rr) terminate = true;
                                }
                            }
                        }
                        if (terminate) break;
                        float3 lightdir, sample_point;
                        lights[light_id]->get_direction(is, lightdir, sample_point);
                        dRay shadow_ray(is.position + is.normal * 0.001f, lightdir);
                        // wf_mat_mix
                        const float3 wo = -ray.d;
                        float3 ext_dir;
                        light_brdf = BRDF_L(lights, bvh->nodes, bvh->tris.data(), is, shadow_ray.d, wo, light_id,
                                            sample_point, ext_dir);
                        ext_brdf = BRDF_f(is, ext_dir, wo);
                        ext_pdf = BRDF_pdf(is, ext_dir, wo);
                        ext_cos = fmaxf(0.0, dot(get_normal(is), ext_dir));
                        ray = dRay(is.position, ext_dir);
                        // wf_shadow
                        light_visible = lights[light_id]->visible(bvh->nodes, bvh->tris.data(), shadow_ray);
                    }
                    ++samples;
                }
                if (out_rgb) {
                    out_rgb[3 * pix] = acc.x;
                    out_rgb[3 * pix + 1] = acc.y;
                    out_rgb[3 * pix + 2] = acc.z;
                }
            }
        }
        n_ext += ext;
        n_sh += g_shadow_calls;
        n_samp += samples;
    };
    auto t1 = std::chrono::steady_clock::now();
    int nt = d->threads > 0 ? d->threads : 1;
    std::vector<std::thread> th;
    for (int k = 1; k < nt; ++k) th.emplace_back(work, k);
    work(0);
    for (auto& x : th) x.join();
    auto t2 = std::chrono::steady_clock::now();
    if (stats) {
        stats[0] = n_ext;
        stats[1] = n_sh;
        stats[2] = n_samp;
    }
    if (ms) {
        ms[0] = std::chrono::duration<double, std::milli>(t2 - t1).count();
        ms[1] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    if (env) ffref_env_free(env);
    if (area) ffref_area_free(area);
    ffref_bvh_free(bvh);
}

void ffref_area_free(void* h)
{
    RefArea* a = (RefArea*)h;
    delete a->light;
    delete a->rect;
    delete a;
}

}  // extern "C"
