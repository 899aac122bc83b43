// ff_cache_render.cu — path tracing with the learned radiance cache.
//
// One frame = one path per pixel plus `train_paths` training paths:
//   k_cached_paths  one thread per path (megakernel: the same vertex code,
//                   ff_paths.cuh, and sampler dimensions as ff_render in
//                   corrected mode).  A pixel path ends at its first rough
//                   vertex after the camera hit and appends a query record
//                   (vertex, throughput, pixel); what it gathered before that
//                   vertex goes to the frame buffer.  A training path, from a
//                   random pixel with its own samples, runs to the full depth
//                   and appends one training record: its first rough vertex
//                   after the camera hit and the radiance the rest of the path
//                   brought back to it (throughput relative to that vertex).
//   train           ff_cache_launch_train over the frame's training records,
//                   in optimiser steps of train_batch records;
//   infer           ff_cache_launch_infer over the queries: frame[pixel] +=
//                   throughput * max(cache, 0);
//   k_frame_to_film the frame joins the film (Kahan-compensated sum, count+1).
// Record counts stay on the device; no host synchronisation inside a frame.
#include <cstring>

#include "ff_cache.cuh"
#include "ff_internal.h"
#include "ff_paths.cuh"
#include "ff_trace.cuh"

namespace {

using namespace ffp;
using ffc::Record;

constexpr int kBlock = 128;

struct CR {
    FFBvhView bvh;
    const FFShadeTri* shade;
    const ff_material* mats;
    const FFTexView* tex;
    const ff_area_light* area;
    FFEnvView env;
    FFLightSet lights;
    ff_camera cam;
    uint32_t W, H, frame, seed, max_depth, rr_depth, n_train;
    int32_t light;
    float shadow_offset, rough_threshold;
    float4* frame_rgb;
    Record* queries;
    uint32_t* n_queries;
    Record* train;
    uint32_t* n_train_out;
    unsigned long long* rays;     // [0] extension, [1] shadow
    unsigned int* err;
};

__device__ __forceinline__ bool is_rough(const FFSurf& s, float threshold)
{
    if (s.kind == FF_MAT_DIFFUSE) return true;
    if (s.kind == FF_MAT_DIELECTRIC) return false;
    return s.roughness >= threshold;
}

__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want)
{
    const uint32_t mask = __ballot_sync(__activemask(), want);
    if (!want) return 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ Record make_record(float3 pos, float rough, float3 wo, float3 n, float3 v, uint32_t pixel)
{
    Record r;
    r.px = pos.x;
    r.py = pos.y;
    r.pz = pos.z;
    r.rough = rough;
    r.wx = wo.x;
    r.wy = wo.y;
    r.wz = wo.z;
    r.v0 = v.x;
    r.nx = n.x;
    r.ny = n.y;
    r.nz = n.z;
    r.v1 = v.y;
    r.pixel = pixel;
    r.v2 = v.z;
    r.pad0 = r.pad1 = 0.f;
    return r;
}

__global__ void __launch_bounds__(kBlock) k_cached_paths(CR a)
{
    __shared__ uint2 s_stack[kShortStack * kBlock];
    FFStack st;
    st.sm = s_stack + threadIdx.x;
    st.stride = kBlock;
    st.sp = 0;
    st.overflow = false;
    const uint32_t npix = a.W * a.H;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool training = i >= npix;
    const bool active = i < npix + a.n_train;
    uint64_t n_ext = 0, n_shadow = 0;
    bool want_query = false, want_train = false;
    Record rec;
    if (active) {
        uint32_t pix, key;
        if (!training) {
            pix = i;
            key = ff_path_key(a.seed, pix, a.frame);
        } else {
            const uint32_t j = i - npix;
            const uint32_t h = ff_wang_hash(ff_wang_hash(a.seed ^ 0x6A09E667u) ^ ff_wang_hash(a.frame * 0x9E3779B9u + j));
            pix = (uint32_t)(((uint64_t)h * npix) >> 32);
            key = ff_path_key(a.seed ^ 0xBB67AE85u, pix, a.frame * a.n_train + j);
        }
        float3 o, d;
        gen_camera_ray(a.cam, (int)a.W, (int)a.H, (int)(pix % a.W), (int)(pix / a.W), rand2(key, 0, DIM_CAM_JITTER),
                       rand2(key, 0, DIM_CAM_LENS), o, d);
        const bool per_vertex = a.lights.light == FF_LIGHT_ALL;
        LightCtx lc = select_light(a.lights, key, 0u);
        float3 beta = make_float3(1.f, 1.f, 1.f);
        float3 beta_rel = make_float3(1.f, 1.f, 1.f);   // throughput since the training vertex
        float3 Lacc = make_float3(0.f, 0.f, 0.f), Ltail = make_float3(0.f, 0.f, 0.f);
        bool tail = false;
        ShadeOut sh;
        bool vis = false, vis_s = false, vis_d = false;
        uint32_t L = 0;
        for (;;) {
            ff_hit hit;
            const bool found = ff_closest_hit(a.bvh, o, d, st, a.err, hit);
            ++n_ext;
            L += 1;
            bool terminate = (L > a.max_depth) || !found;
            if (!found && L == 1) Lacc = Lacc + beta * env_L(a.env, d, true);
            if (L > 1) {
                float3 lb = make_float3(0.f, 0.f, 0.f);
                if (vis) lb = lb + sh.c_nee;
                if (vis_s) lb = lb + sh.c_spec;
                if (vis_d) lb = lb + sh.c_diff;
                if (tail) Ltail = Ltail + lb * beta_rel;
                else Lacc = Lacc + lb * beta;
                if (sh.ext_f == make_float3(0.f, 0.f, 0.f) || sh.ext_pdf == 0.f) {
                    terminate = true;
                } else {
                    const float3 fc = (sh.ext_f * sh.ext_cos) / sh.ext_pdf;
                    beta *= fc;
                    beta_rel *= fc;
                    if (L > a.rr_depth) {
                        const float q = hmax(0.05f, 1.f - beta.y);
                        if (ff_rand(key, dim_of(L, DIM_RR)) < q || q >= 1.f) {
                            terminate = true;
                        } else {
                            beta = beta / (1.f - q);
                            beta_rel = beta_rel / (1.f - q);
                        }
                    }
                }
            }
            if (terminate) break;
            const FFShadeTri& t = a.shade[hit.prim];
            const float u = hit.u, v = hit.v;
            const float3 n = normalize3(u * t.n1 + v * t.n2 + ((1.f - u) - v) * t.n0);
            const float3 pos = o + hit.t * d;
            const float wuv = (1.f - u) - v;
            const float2 tuv = make_float2(u * t.uv1.x + v * t.uv2.x + wuv * t.uv0.x,
                                           u * t.uv1.y + v * t.uv2.y + wuv * t.uv0.y);
            const ff_material& mm = a.mats[t.material];
            const FFSurf surf = resolve_surface(mm, a.tex, tuv);
            const float3 wo = -d;
            if (L >= 2 && !tail && is_rough(surf, a.rough_threshold)) {
                if (!training) {
                    // the cache answers for everything from this vertex on
                    rec = make_record(pos, surf.roughness, wo, n, beta, pix);
                    want_query = true;
                    break;
                }
                rec = make_record(pos, surf.roughness, wo, n, make_float3(0.f, 0.f, 0.f), pix);
                tail = true;
                want_train = true;
                beta_rel = make_float3(1.f, 1.f, 1.f);
            }
            float3 wi, sp;
            if (per_vertex) lc = select_light(a.lights, key, L);
            sample_light(lc, pos, key, L, wi, sp);
            sh.c_spec = sh.c_diff = make_float3(0.f, 0.f, 0.f);
            switch (surf.kind) {
                case FF_MAT_MIX: shade_mix(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, sp, key, L, sh); break;
                case FF_MAT_DIFFUSE: shade_diffuse(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
                case FF_MAT_CONDUCTOR: shade_conductor(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
                case FF_MAT_DIELECTRIC: shade_dielectric(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
                default: shade_coat(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
            }
            const float3 lo = pos + n * a.shadow_offset;
            sh.ray_nee = light_vis_ray(lc, lo, wi, key, L, DIM_NEE_VIS, sh.r_nee);
            vis = sh.ray_nee && !ff_occluded(a.bvh, sh.r_nee, st, a.err);
            vis_s = sh.ray_spec && !ff_occluded(a.bvh, sh.r_spec, st, a.err);
            vis_d = sh.ray_diff && !ff_occluded(a.bvh, sh.r_diff, st, a.err);
            n_shadow += (sh.ray_nee ? 1 : 0) + (sh.ray_spec ? 1 : 0) + (sh.ray_diff ? 1 : 0);
            const float side = dot3(sh.ext_d, n) >= 0.f ? 1.f : -1.f;
            o = pos + n * (side * a.shadow_offset);
            d = sh.ext_d;
        }
        if (!training) a.frame_rgb[pix] = make_float4(Lacc.x, Lacc.y, Lacc.z, 0.f);
        if (want_train) {
            rec.v0 = Ltail.x;
            rec.v1 = Ltail.y;
            rec.v2 = Ltail.z;
            want_train = isfinite(Ltail.x) && isfinite(Ltail.y) && isfinite(Ltail.z);
        }
    }
    const uint32_t qs = warp_append(a.n_queries, want_query);
    if (want_query) a.queries[qs] = rec;
    const uint32_t ts = warp_append(a.n_train_out, want_train);
    if (want_train) a.train[ts] = rec;
    for (int off = 16; off; off >>= 1) {
        n_ext += __shfl_down_sync(0xffffffffu, n_ext, off);
        n_shadow += __shfl_down_sync(0xffffffffu, n_shadow, off);
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(a.rays, (unsigned long long)n_ext);
        atomicAdd(a.rays + 1, (unsigned long long)n_shadow);
    }
}

__device__ __forceinline__ void kahan(float& sum, float& comp, float x)
{
    const float y = x - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

__global__ void k_frame_to_film(const float4* __restrict__ frame, uint32_t n, float4* __restrict__ acc,
                                float4* __restrict__ comp, uint32_t* __restrict__ cnt, const uint32_t* __restrict__ rec_cnt,
                                unsigned long long* __restrict__ rec_total)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        rec_total[0] += rec_cnt[0];
        rec_total[1] += rec_cnt[1];
    }
    if (i >= n) return;
    const float4 f = frame[i];
    float4 s = acc[i], c = comp[i];
    kahan(s.x, c.x, f.x);
    kahan(s.y, c.y, f.y);
    kahan(s.z, c.z, f.z);
    acc[i] = s;
    comp[i] = c;
    cnt[i] += 1u;
}

}  // namespace

void ff_cached_render(ff_context* ctx, ff_scene* scene, ff_cache* c, const ff_render_settings* st, ff_film* film,
                      ff_render_stats* stats)
{
    FF_REQUIRE(st->spp > 0 && st->max_depth >= 1 && st->max_depth <= 64, "spp > 0, 1 <= max_depth <= 64");
    ff_check_light(scene, st->light, FF_MODE_CORRECTED);
    const uint32_t W = film->width, H = film->height, npix = W * H;
    const uint32_t n_train = c->prm.train_paths;
    const uint32_t batch = c->prm.train_batch ? c->prm.train_batch : (n_train ? n_train : 1u);
    cudaStream_t stream = ctx->stream;
    if (c->ws_pixels < npix) {
        c->queries.alloc(sizeof(Record) * (size_t)npix);
        c->frame.alloc(sizeof(float4) * (size_t)npix);
        c->ws_pixels = npix;
    }
    if (c->ws_train < n_train) {
        c->train_recs.alloc(sizeof(Record) * (size_t)n_train);
        c->ws_train = n_train;
    }
    c->counters.alloc(64);
    FF_CUDA_CHECK(cudaMemsetAsync(c->counters.ptr, 0, 64, stream));
    uint32_t* cnt = c->counters.as<uint32_t>();            // [0] queries, [1] training records
    unsigned long long* rays = reinterpret_cast<unsigned long long*>(c->counters.as<char>() + 16);
    unsigned int* err = reinterpret_cast<unsigned int*>(c->counters.as<char>() + 32);
    unsigned long long* totals = reinterpret_cast<unsigned long long*>(c->counters.as<char>() + 48);
    CR a;
    a.bvh = scene->view();
    a.shade = scene->shade.as<FFShadeTri>();
    a.mats = scene->materials.as<ff_material>();
    a.tex = scene->tex_table.as<FFTexView>();
    a.area = scene->area_lights.as<ff_area_light>();
    a.env = ff_env_view(scene);
    a.lights = ff_light_set(scene, st->light, FF_MODE_CORRECTED);
    a.cam = scene->camera;
    a.W = W;
    a.H = H;
    a.seed = st->seed;
    a.max_depth = st->max_depth;
    a.rr_depth = st->rr_depth;
    a.n_train = n_train;
    a.light = st->light;
    a.shadow_offset = st->shadow_offset > 0.f ? st->shadow_offset : 0.001f;
    a.rough_threshold = c->prm.rough_threshold;
    a.frame_rgb = c->frame.as<float4>();
    a.queries = c->queries.as<Record>();
    a.n_queries = cnt;
    a.train = c->train_recs.as<Record>();
    a.n_train_out = cnt + 1;
    a.rays = rays;
    a.err = err;
    const uint32_t blocks = (npix + n_train + kBlock - 1) / kBlock;
    const bool profile = (st->flags & FF_RENDER_PROFILE) != 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    if (profile)
        for (auto& e : ev) FF_CUDA_CHECK(cudaEventCreate(&e));
    float ms_paths = 0.f, ms_train = 0.f, ms_query = 0.f;
    uint64_t launches = 0;
    FF_CUDA_CHECK(cudaEventRecord(ctx->ev0, stream));
    for (uint32_t f = 0; f < st->spp; ++f) {
        a.frame = st->sample_offset + f;
        FF_CUDA_CHECK(cudaMemsetAsync(cnt, 0, 8, stream));
        if (profile) FF_CUDA_CHECK(cudaEventRecord(ev[0], stream));
        k_cached_paths<<<blocks, kBlock, 0, stream>>>(a);
        launches += 1;
        if (profile) FF_CUDA_CHECK(cudaEventRecord(ev[1], stream));
        for (uint32_t off = 0; off < n_train; off += batch) {
            ff_cache_launch_train_slice(c, a.train, off, std::min(batch, n_train - off), cnt + 1);
            launches += 3;
        }
        if (profile) FF_CUDA_CHECK(cudaEventRecord(ev[2], stream));
        ff_cache_launch_infer(c, a.queries, npix, cnt, nullptr, a.frame_rgb);
        k_frame_to_film<<<(npix + 255) / 256, 256, 0, stream>>>(a.frame_rgb, npix, film->accum.as<float4>(),
                                                                 film->comp.as<float4>(), film->count.as<uint32_t>(),
                                                                 cnt, totals);
        launches += 2;
        FF_CUDA_CHECK(cudaGetLastError());
        if (profile) {
            FF_CUDA_CHECK(cudaEventRecord(ev[3], stream));
            FF_CUDA_CHECK(cudaEventSynchronize(ev[3]));
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[0], ev[1]);
            ms_paths += t;
            cudaEventElapsedTime(&t, ev[1], ev[2]);
            ms_train += t;
            cudaEventElapsedTime(&t, ev[2], ev[3]);
            ms_query += t;
        }
    }
    if (profile)
        for (auto& e : ev) cudaEventDestroy(e);
    FF_CUDA_CHECK(cudaEventRecord(ctx->ev1, stream));
    unsigned long long h[6] = {0, 0, 0, 0, 0, 0};
    FF_CUDA_CHECK(cudaMemcpyAsync(h, c->counters.as<char>() + 16, sizeof(h), cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaStreamSynchronize(stream));
    if ((unsigned int)h[2]) throw FFError{FF_ERR_INTERNAL, "traversal exceeded its step bound (malformed BVH)"};
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->extension_rays = h[0];
        stats->shadow_rays = h[1];
        stats->samples = (uint64_t)npix * st->spp;
        stats->frames = st->spp;
        stats->ms_total = ms;
        stats->kernel_launches = launches;
        stats->ms_cache_paths = ms_paths;
        stats->ms_cache_train = ms_train;
        stats->ms_cache_query = ms_query;
        stats->cache_queries = h[4];
        stats->cache_records = h[5];
    }
}
