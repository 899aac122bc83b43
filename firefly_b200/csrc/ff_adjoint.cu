// ff_adjoint.cu — path-replay adjoint of the path tracer (no reference
// counterpart: the reference renders only).
//
// For a loss L(I) of the mean-radiance image I, given dL/dI per pixel, the
// adjoint accumulates dL/d(texel) of one albedo texture and of the
// environment map.  One thread per pixel sample, the path computed exactly as
// ff_render computes it in corrected mode (same sampler dimensions, same
// shading code, ff_paths.cuh):
//   pass 1  trace the path and sum its radiance L_s;
//   pass 2  replay it from the same seed (path replay backpropagation:
//           nothing is stored per vertex) and, at every vertex k whose albedo
//           a_k comes from the texture, add dL/dI * L_{>=k} / a_k to the
//           texels of its bilinear footprint, L_{>=k} = L_s - (radiance added
//           before vertex k); at every NEE and camera-miss lookup of the
//           environment, add dL/dI * (contribution / radiance looked up) to
//           the env texels of the lookup's footprint.
// ff_render_adjoint runs the replay on the wavefront stages by default
// (ff_wavefront_adjoint, ff_wavefront.cu: the same k_logic / k_shade /
// k_trace stages as ff_render, one slot per path, primal pass then replay of
// the same sample).  This file holds the one-thread-per-sample megakernel
// variants: the replay (FF_ADJOINT_MEGAKERNEL, kept as a cross-check) and the
// store-all variant, which keeps the vertices of pass 1 in local memory and
// needs no replay; it is the reference both replays are checked against.
// Sampling is detached: the importance tables and the Russian-roulette
// probability are not differentiated.  Gradients reach albedo textures of
// FF_MAT_DIFFUSE surfaces (their BRDF is linear in the albedo), roughness
// textures of the GGX surfaces (mixed, conductor, rough dielectric, coat:
// at vertex k, dI . [d(own terms)/dr + L_{>k} * dlog(ext_f)/dr] with
// L_{>k} = L_s - (radiance up to and including vertex k's own terms), the
// directions, pdfs and MIS weights held at their sampled values) and the
// environment through camera misses and the NEE term.
// Scatter: texel gradients go to global memory with atomicAdd after a
// warp-level pre-reduction of lanes that hit the same texel (__match_any_sync).
#include "ff_internal.h"
#include "ff_adjoint.cuh"
#include "ff_paths.cuh"
#include "ff_trace.cuh"

namespace {

using namespace ffp;
using namespace ffadj;

constexpr int kAdjBlock = 128;
constexpr int kMaxVerts = 16;

struct ADJ {
    FFBvhView bvh;
    const FFShadeTri* shade;
    const FFTangentTri* tan;
    const ff_material* mats;
    const FFTexView* tex;
    const ff_area_light* area;
    FFEnvView env;
    FFLightSet lights;
    ff_camera cam;
    uint32_t W, H, spp, sample_offset, seed, max_depth, rr_depth;
    int32_t light;
    float shadow_offset;
    const float* d_image;   // W*H*3
    int32_t texture;        // texture receiving gradients, -1 none
    float* grad_tex;        // texels*3
    float* grad_env;        // env texels*3 or nullptr
    int32_t rough_texture;  // roughness texture receiving gradients (channel x), -1 none
    float* grad_rough;      // texels*3 of rough_texture (channel x written) or nullptr
    unsigned long long* rays;
    unsigned int* err;
};

// The traversals and the shading switch are called, not inlined: each is one
// copy of its code however many sites use it.
__device__ __noinline__ bool closest_hit(const FFBvhView bvh, unsigned int* err, float3 o, float3 d, bool two,
                                         FFStack& st, ff_hit& h)
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

__device__ __noinline__ bool occluded(const FFBvhView bvh, unsigned int* err, const ff_ray ray, FFStack& st)
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

__device__ __noinline__ void shade_vertex(const LightCtx& lc, const FFSurf& surf, float3 pos, float3 n, float3 wo,
                                          float3 wi, float3 sp, uint32_t key, uint32_t L, bool back, ShadeOut& sh)
{
    sh.c_spec = sh.c_diff = make_float3(0.f, 0.f, 0.f);
    switch (surf.kind) {
        case FF_MAT_MIX: shade_mix<true>(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, sp, key, L, sh); break;
        case FF_MAT_DIFFUSE: shade_diffuse<true>(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
        case FF_MAT_CONDUCTOR: shade_conductor<true>(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
        case FF_MAT_DIELECTRIC: shade_dielectric(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, back, sh); break;
        default: shade_coat(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
    }
}

struct VertexRec {
    float3 a;           // albedo at the vertex (texture-fed diffuse only)
    float3 L_before;    // radiance added before the vertex's terms
    float u, v;         // texcoords
    bool albedo;        // the vertex takes an albedo gradient
    bool rough;         // the vertex takes a roughness gradient
    int8_t rough_ch;    // channel of the roughness texture it reads (0 or 1)
    float g_imm;        // dI . d(own terms)/dr
    float3 dext;        // d/dr log(ext_f)
    float3 L_after;     // radiance added up to and including the vertex's own terms
};

// One path sample.  mode 0: primal (returns L_s).  mode 1: replay with
// gradients (L_total = L_s of pass 1).  mode 2 (STORE_ALL only): primal that
// records the vertices into rec.  ROUGH: roughness gradients requested (a
// separate instantiation keeps the albedo/environment kernel's registers).
// The mode is a run-time value and the kernel calls this function from one
// site (a loop over the passes), and the shadow rays are traced from one
// site (a loop over the three rays), so the kernel holds one copy of the
// shading code and two of the traversal: with a copy per pass and per ray
// the code outgrew the instruction cache (instruction-fetch stalls were the
// largest stall reason).
template <bool STORE_ALL, bool ROUGH>
__device__ __forceinline__ float3 run_path(const ADJ& a, const int mode, uint32_t pix, uint32_t sample, FFStack& st,
                                           float3 L_total, float3 dI, VertexRec* rec, int* n_rec, uint64_t& rays,
                                           uint64_t& atom, uint64_t& atom_r)
{
    const bool grad = mode != 0;
    const bool record = STORE_ALL && mode == 2;
    const uint32_t key = ff_path_key(a.seed, pix, sample);
    float3 o, d;
    gen_camera_ray(a.cam, (int)a.W, (int)a.H, (int)(pix % a.W), (int)(pix / a.W), rand2(key, 0, DIM_CAM_JITTER),
                   rand2(key, 0, DIM_CAM_LENS), o, d);
    const LightCtx lc = select_light(a.lights, key, 0u);   // a fixed light (FF_LIGHT_ALL is rejected)
    float3 beta = make_float3(1.f, 1.f, 1.f);
    float3 Lacc = make_float3(0.f, 0.f, 0.f);
    ShadeOut sh;
    bool vis = false, vis_s = false, vis_d = false;
    float3 nee_env_coef = make_float3(0.f, 0.f, 0.f), nee_dir = make_float3(0.f, 0.f, 0.f);
    uint32_t L = 0;
    bool inside = false;   // the ray runs inside an object: traced two-sided
    for (;;) {
        ff_hit hit;
        const bool found = closest_hit(a.bvh, a.err, o, d, inside, st, hit);
        ++rays;
        L += 1;
        bool terminate = (L > a.max_depth) || !found;
        if (!found && L == 1) {
            const float3 Le = env_L(a.env, d, true);
            const float3 c = beta * Le;
            if (grad && a.grad_env && a.env.rgb) {
                float3 dd = d;
                dd.y = clampf(dd.y, -1.f, 1.f);
                const float2 uv = spherical_map(dd);
                atom += scatter_footprint(a.grad_env, footprint(a.env.width, a.env.height, uv.x, uv.y), dI * beta);
            }
            Lacc = Lacc + c;
        }
        if (L > 1) {
            float3 lb = make_float3(0.f, 0.f, 0.f);
            if (vis) lb = lb + sh.c_nee;
            if (vis_s) lb = lb + sh.c_spec;
            if (vis_d) lb = lb + sh.c_diff;
            if (vis || vis_s || vis_d) {
                if (grad && vis && a.grad_env && lc.is_env && a.env.rgb) {
                    // NEE term c_nee = coef * Le(wl): d/dLe = beta * coef
                    const float2 uv = spherical_map(nee_dir);
                    atom += scatter_footprint(a.grad_env, footprint(a.env.width, a.env.height, uv.x, uv.y),
                                      dI * beta * nee_env_coef);
                }
                Lacc = Lacc + lb * beta;
            }
            if (sh.ext_f == make_float3(0.f, 0.f, 0.f) || sh.ext_pdf == 0.f) {
                terminate = true;
            } else {
                beta *= (sh.ext_f * sh.ext_cos) / sh.ext_pdf;
                if (L > a.rr_depth) {
                    const float q = hmax(0.05f, 1.f - beta.y);
                    if (ff_rand(key, dim_of(L, DIM_RR)) < q) terminate = true;
                    else if (q >= 1.f) terminate = true;
                    else beta = beta / (1.f - q);
                }
            }
        }
        if (terminate) break;
        // hit attributes
        const bool back = hit_back(hit.prim);   // hit from inside an object
        const uint32_t prim = hit_index(hit.prim);
        const FFShadeRec t = ff_load_shade(a.shade, prim);
        const float u = hit.u, v = hit.v;
        // ng: the interpolated normal the ray offsets follow (kernel.cu:437);
        // n: the shading normal (get_normal: a normal texture's frame, else ng);
        // both face the ray
        float3 ng = normalize3(u * t.n1 + v * t.n2 + ((1.f - u) - v) * t.n0);
        const float3 pos = o + hit.t * d;
        const float wuv = (1.f - u) - v;
        const float2 tuv = make_float2(u * t.uv1.x + v * t.uv2.x + wuv * t.uv0.x, u * t.uv1.y + v * t.uv2.y + wuv * t.uv0.y);
        const ff_material& mm = a.mats[t.material];
        float3 n = shading_normal(mm, a.tex, a.tan, prim, u, v, tuv, ng);
        if (back) {
            ng = -ng;
            n = -n;
        }
        float3 wi, sp;
        sample_light(lc, pos, key, L, wi, sp);
        const FFSurf surf = resolve_surface(mm, a.tex, tuv);
        const float3 wo = -d;
        shade_vertex(lc, surf, pos, n, wo, wi, sp, key, L, back, sh);
        const bool diel = surf.kind == FF_MAT_DIELECTRIC;
        const float3 lo = pos + ng * (((diel && dot3(wi, ng) < 0.f) ? -1.f : 1.f) * a.shadow_offset);
        sh.ray_nee = light_vis_ray(lc, lo, wi, key, L, DIM_NEE_VIS, sh.r_nee);
        uint32_t visible = 0;
#pragma unroll 1
        for (int k = 0; k < 3; ++k) {
            const bool want = k == 0 ? sh.ray_nee : (k == 1 ? sh.ray_spec : sh.ray_diff);
            if (!want) continue;
            const ff_ray r = k == 0 ? sh.r_nee : (k == 1 ? sh.r_spec : sh.r_diff);
            if (!occluded(a.bvh, a.err, r, st)) visible |= 1u << k;
            ++rays;
        }
        vis = (visible & 1u) != 0;
        vis_s = (visible & 2u) != 0;
        vis_d = (visible & 4u) != 0;
        // d(c_nee)/d(Le) for the environment gradient: c_nee is linear in Le(wi)
        nee_dir = wi;
        nee_dir.y = clampf(nee_dir.y, -1.f, 1.f);
        {
            const float3 Li = light_L(lc, wi);
            nee_env_coef = make_float3(Li.x != 0.f ? sh.c_nee.x / Li.x : 0.f, Li.y != 0.f ? sh.c_nee.y / Li.y : 0.f,
                                       Li.z != 0.f ? sh.c_nee.z / Li.z : 0.f);
        }
        const bool tex_grad = surf.kind == FF_MAT_DIFFUSE && mm.base_color_tex >= 0 && mm.base_color_tex == a.texture;
        // roughness gradient: GGX surfaces whose roughness comes from the
        // texture (above the 0.01 floor of resolve_surface, where it is flat)
        const int rch = ROUGH && grad && surf.kind != FF_MAT_DIFFUSE ? rough_channel(mm, a.rough_texture) : -1;
        const bool rough_grad = rch >= 0 && surf.roughness > 0.01f;
        RoughTerms rt;
        float3 rimm = make_float3(0.f, 0.f, 0.f);
        float3 L_after = Lacc;
        if (rough_grad) {
            rt = rough_terms(sh, n, wo, wi, surf.roughness, diel);
            rimm = rough_own(rt, vis, vis_s, beta);
            float3 own = make_float3(0.f, 0.f, 0.f);
            if (vis) own = own + sh.c_nee;
            if (vis_s) own = own + sh.c_spec;
            if (vis_d) own = own + sh.c_diff;
            L_after = Lacc + own * beta;
        }
        if (mode == 1 && rough_grad) {
            const float3 Lgt = L_total - L_after;
            const float g = dot3(dI, rimm + Lgt * rt.dext);
            const FFTexView tv = a.tex[a.rough_texture];
            atom_r += scatter_footprint1(a.grad_rough, footprint(tv.width, tv.height, tuv.x, tuv.y), g, rch);
        }
        if (mode == 1 && tex_grad) {
            const FFTexView tv = a.tex[a.texture];
            atom += scatter_footprint(a.grad_tex, footprint(tv.width, tv.height, tuv.x, tuv.y),
                                      albedo_grad(L_total - Lacc, surf.albedo, dI));
        }
        if (record && (tex_grad || rough_grad) && *n_rec < kMaxVerts) {
            VertexRec& r = rec[(*n_rec)++];
            r.a = surf.albedo;
            r.L_before = Lacc;
            r.u = tuv.x;
            r.v = tuv.y;
            r.albedo = tex_grad;
            r.rough = rough_grad;
            r.rough_ch = (int8_t)rch;
            if (rough_grad) {
                r.g_imm = dot3(dI, rimm);
                r.dext = rt.dext;
                r.L_after = L_after;
            }
        }
        const float side = dot3(sh.ext_d, ng) >= 0.f ? 1.f : -1.f;
        o = pos + ng * (side * a.shadow_offset);
        d = sh.ext_d;
        inside = runs_inside(back, diel, side);
    }
    return Lacc;
}

template <bool STORE_ALL, bool ROUGH>
__global__ void __launch_bounds__(kAdjBlock) k_adjoint(ADJ a)
{
    __shared__ uint2 s_stack[kShortStack * kAdjBlock];
    FFStack st;
    st.sm = s_stack + threadIdx.x;
    st.stride = kAdjBlock;
    st.sp = 0;
    st.overflow = false;
    const uint64_t n = (uint64_t)a.W * a.H * a.spp;
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t rays = 0, atom = 0, atom_r = 0;
    if (i < n) {
        const uint32_t pix = (uint32_t)(i % ((uint64_t)a.W * a.H));
        const uint32_t sample = a.sample_offset + (uint32_t)(i / ((uint64_t)a.W * a.H));
        const float inv_spp = 1.f / (float)a.spp;
        const float3 dI = make_float3(a.d_image[3 * (size_t)pix] * inv_spp, a.d_image[3 * (size_t)pix + 1] * inv_spp,
                                      a.d_image[3 * (size_t)pix + 2] * inv_spp);
        if (!STORE_ALL) {
            float3 Ls = make_float3(0.f, 0.f, 0.f);
#pragma unroll 1
            for (int pass = 0; pass < 2; ++pass) {
                const float3 Lp = run_path<false, ROUGH>(a, pass, pix, sample, st, Ls, dI, nullptr, nullptr, rays, atom,
                                                         atom_r);
                if (pass == 0) Ls = Lp;
            }
        } else {
            VertexRec rec[kMaxVerts];
            int n_rec = 0;
            const float3 Ls =
                run_path<true, ROUGH>(a, 2, pix, sample, st, make_float3(0.f, 0.f, 0.f), dI, rec, &n_rec, rays, atom,
                                      atom_r);
            for (int k = 0; k < n_rec; ++k) {
                const VertexRec& r = rec[k];
                if (ROUGH && r.rough) {
                    const float g = r.g_imm + dot3(dI, (Ls - r.L_after) * r.dext);
                    const FFTexView tv = a.tex[a.rough_texture];
                    atom_r += scatter_footprint1(a.grad_rough, footprint(tv.width, tv.height, r.u, r.v), g, r.rough_ch);
                }
                if (!r.albedo) continue;
                const FFTexView tv = a.tex[a.texture];
                atom += scatter_footprint(a.grad_tex, footprint(tv.width, tv.height, r.u, r.v),
                                          albedo_grad(Ls - r.L_before, r.a, dI));
            }
        }
    }
    // per-warp ray count
    for (int off = 16; off; off >>= 1) {
        rays += __shfl_down_sync(0xffffffffu, rays, off);
        atom += __shfl_down_sync(0xffffffffu, atom, off);
        atom_r += __shfl_down_sync(0xffffffffu, atom_r, off);
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(a.rays, (unsigned long long)rays);
        atomicAdd(a.rays + 2, (unsigned long long)atom);
        if (atom_r) atomicAdd(a.rays + 3, (unsigned long long)atom_r);
    }
}

}  // namespace

void ff_adjoint_render(ff_context* ctx, ff_scene* scene, const ff_render_settings* st, const ff_adjoint_desc* ad,
                       ff_render_stats* stats)
{
    FF_REQUIRE(ad->width > 0 && ad->height > 0 && ad->d_image, "adjoint image required");
    const bool store_all = (ad->flags & FF_ADJOINT_STORE_ALL) != 0;
    const bool mega = store_all || (ad->flags & FF_ADJOINT_MEGAKERNEL) != 0;
    FF_REQUIRE(st->spp > 0 && st->max_depth >= 1, "spp > 0 and max_depth >= 1 required");
    FF_REQUIRE(!mega || st->max_depth < (uint32_t)kMaxVerts, "the megakernel variants take max_depth < 16");
    FF_REQUIRE(ad->texture < (int32_t)scene->textures.size(), "texture index out of range");
    FF_REQUIRE(ad->texture < 0 || ad->grad_texture, "grad_texture required for a texture gradient");
    FF_REQUIRE(st->light != FF_LIGHT_ALL, "the adjoint needs one light (FF_LIGHT_ALL is not supported)");
    ff_check_light(scene, st->light, FF_MODE_CORRECTED);
    cudaStream_t stream = ctx->stream;
    const bool dev = (ad->flags & FF_MEM_DEVICE) != 0;
    const size_t npix = (size_t)ad->width * ad->height;
    const bool rough = ad->grad_roughness != nullptr;
    FF_REQUIRE(!rough || (ad->roughness_texture >= 0 && ad->roughness_texture < (int32_t)scene->textures.size()),
               "roughness_texture out of range");
    auto texels = [&](int32_t t) {
        FFTexView v;
        FF_CUDA_CHECK(cudaMemcpy(&v, scene->tex_table.as<FFTexView>() + t, sizeof(v), cudaMemcpyDeviceToHost));
        return (size_t)v.width * v.height;
    };
    const size_t ntex = ad->texture >= 0 ? (size_t)3 * texels(ad->texture) : 0;
    const size_t nrough = rough ? (size_t)3 * texels(ad->roughness_texture) : 0;
    const size_t nenv = (size_t)3 * scene->env.width * scene->env.height;
    // staging of host buffers and the counters, kept on the context between
    // calls (calls on one context are externally synchronised)
    DevBuf &dimg = ctx->adj_io[0], &gtex = ctx->adj_io[1], &genv = ctx->adj_io[2], &grough = ctx->adj_io[3],
           &ctr = ctx->adj_io[4];
    const float* d_image = ad->d_image;
    float* g_tex = ad->grad_texture;
    float* g_env = ad->grad_env;
    float* g_rough = ad->grad_roughness;
    if (!dev) {
        dimg.alloc(sizeof(float) * 3 * npix);
        FF_CUDA_CHECK(cudaMemcpyAsync(dimg.ptr, ad->d_image, sizeof(float) * 3 * npix, cudaMemcpyHostToDevice, stream));
        d_image = dimg.as<float>();
        if (ntex) {
            gtex.alloc(sizeof(float) * ntex);
            FF_CUDA_CHECK(cudaMemcpyAsync(gtex.ptr, ad->grad_texture, sizeof(float) * ntex, cudaMemcpyHostToDevice, stream));
            g_tex = gtex.as<float>();
        }
        if (ad->grad_env && nenv) {
            genv.alloc(sizeof(float) * nenv);
            FF_CUDA_CHECK(cudaMemcpyAsync(genv.ptr, ad->grad_env, sizeof(float) * nenv, cudaMemcpyHostToDevice, stream));
            g_env = genv.as<float>();
        }
        if (nrough) {
            grough.alloc(sizeof(float) * nrough);
            FF_CUDA_CHECK(cudaMemcpyAsync(grough.ptr, ad->grad_roughness, sizeof(float) * nrough,
                                          cudaMemcpyHostToDevice, stream));
            g_rough = grough.as<float>();
        }
    }
    ctr.alloc(64);
    FF_CUDA_CHECK(cudaMemsetAsync(ctr.ptr, 0, 64, stream));
    ADJ a;
    a.bvh = scene->view();
    a.shade = scene->shade.as<FFShadeTri>();
    a.tan = scene->tangent.as<FFTangentTri>();
    a.mats = scene->materials.as<ff_material>();
    a.tex = scene->tex_table.as<FFTexView>();
    a.area = scene->area_lights.as<ff_area_light>();
    a.env = ff_env_view(scene);
    a.lights = ff_light_set(scene, st->light, FF_MODE_CORRECTED);
    a.cam = scene->camera;
    a.W = ad->width;
    a.H = ad->height;
    a.spp = st->spp;
    a.sample_offset = st->sample_offset;
    a.seed = st->seed;
    a.max_depth = st->max_depth;
    a.rr_depth = st->rr_depth;
    a.light = st->light;
    a.shadow_offset = st->shadow_offset > 0.f ? st->shadow_offset : 0.001f;
    a.d_image = d_image;
    a.texture = ad->texture;
    a.grad_tex = g_tex;
    a.grad_env = (ad->grad_env && nenv) ? g_env : nullptr;
    a.rough_texture = rough ? ad->roughness_texture : -1;
    a.grad_rough = rough ? g_rough : nullptr;
    a.rays = ctr.as<unsigned long long>();
    a.err = reinterpret_cast<unsigned int*>(ctr.as<char>() + 8);
    const uint64_t n = (uint64_t)npix * st->spp;
    const uint64_t blocks = (n + kAdjBlock - 1) / kAdjBlock;
    FF_REQUIRE(!mega || blocks < (1ull << 31), "adjoint launch too large");
    FF_CUDA_CHECK(cudaEventRecord(ctx->ev0, stream));
    if (!mega) {
        // the default: path replay on the wavefront stages
        FFAdjointTarget t{ad->width, ad->height, d_image, ad->texture, ntex ? g_tex : nullptr, a.grad_env,
                          a.rough_texture, a.grad_rough, ctr.as<unsigned long long>() + 2};
        ff_wavefront_adjoint(ctx, scene, st, t, stats);
    } else if (store_all && rough) {
        k_adjoint<true, true><<<(unsigned)blocks, kAdjBlock, 0, stream>>>(a);
    } else if (store_all) {
        k_adjoint<true, false><<<(unsigned)blocks, kAdjBlock, 0, stream>>>(a);
    } else if (rough) {
        k_adjoint<false, true><<<(unsigned)blocks, kAdjBlock, 0, stream>>>(a);
    } else {
        k_adjoint<false, false><<<(unsigned)blocks, kAdjBlock, 0, stream>>>(a);
    }
    FF_CUDA_CHECK(cudaGetLastError());
    FF_CUDA_CHECK(cudaEventRecord(ctx->ev1, stream));
    if (!dev) {
        if (ntex)
            FF_CUDA_CHECK(cudaMemcpyAsync(ad->grad_texture, g_tex, sizeof(float) * ntex, cudaMemcpyDeviceToHost, stream));
        if (ad->grad_env && nenv)
            FF_CUDA_CHECK(cudaMemcpyAsync(ad->grad_env, g_env, sizeof(float) * nenv, cudaMemcpyDeviceToHost, stream));
        if (nrough)
            FF_CUDA_CHECK(cudaMemcpyAsync(ad->grad_roughness, g_rough, sizeof(float) * nrough, cudaMemcpyDeviceToHost,
                                          stream));
    }
    unsigned long long h_ctr[4] = {0, 0, 0, 0};
    FF_CUDA_CHECK(cudaMemcpyAsync(h_ctr, ctr.ptr, sizeof(h_ctr), cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaStreamSynchronize(stream));
    if ((unsigned int)h_ctr[1]) throw FFError{FF_ERR_INTERNAL, "traversal exceeded its step bound (malformed BVH)"};
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        // the megakernel counts every traced ray (both passes) in h_ctr[0];
        // the wavefront fills extension_rays / shadow_rays itself
        if (mega) {
            stats->extension_rays = h_ctr[0];
            stats->kernel_launches = 1;
        }
        stats->grad_atomics = h_ctr[2];
        stats->grad_atomics_roughness = h_ctr[3];
        stats->samples = n;
        stats->ms_total = ms;
    }
}

namespace {

// One Adam step (Kingma & Ba 2015) with bias correction, then a clamp of the
// parameter to [lo, hi]: m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// p -= lr * (m / (1-b1^t)) / (sqrt(v / (1-b2^t)) + eps).
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       uint64_t n, float lr, float b1, float b2, float eps, float c1, float c2, float lo, float hi)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float step = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = fminf(fmaxf(p[i] - step, lo), hi);
}

}  // namespace

extern "C" ff_status ff_optimizer_adam_step(ff_context* ctx, float* param, const float* grad, float* m, float* v,
                                            uint64_t n, const ff_adam_params* hp)
{
    if (!ctx || !param || !grad || !m || !v || !hp) return FF_ERR_INVALID_ARG;
    if (n == 0) return FF_OK;
    try {
        FF_CUDA_CHECK(cudaSetDevice(ctx->device));
        FF_REQUIRE(hp->step >= 1, "Adam step counts from 1");
        const float c1 = 1.f - powf(hp->beta1, (float)hp->step);
        const float c2 = 1.f - powf(hp->beta2, (float)hp->step);
        const uint64_t blocks = (n + 255) / 256;
        FF_REQUIRE(blocks < (1ull << 31), "parameter vector too large");
        k_adam<<<(unsigned)blocks, 256, 0, ctx->stream>>>(param, grad, m, v, n, hp->lr, hp->beta1, hp->beta2, hp->eps,
                                                         c1, c2, hp->lo, hp->hi);
        FF_CUDA_CHECK(cudaGetLastError());
        return FF_OK;
    } catch (const FFError& e) {
        ctx->last_error = e.msg;
        return e.status;
    }
}
