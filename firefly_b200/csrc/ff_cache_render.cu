// ff_cache_render.cu — path tracing with the learned radiance cache.
//
// One frame = one path per pixel plus `train_paths` training paths:
//   k_training_paths  one thread per training path (megakernel: the same
//                     vertex code, ff_paths.cuh, and sampler as ff_render in
//                     corrected mode), from a random pixel with its own
//                     samples, to the full depth; it appends one training
//                     record: its first rough vertex after the camera hit and
//                     the radiance the rest of the path brought back to it
//                     (throughput relative to that vertex);
//   train             ff_cache_launch_train over the frame's records, in
//                     optimiser steps of train_batch records;
//   pixel paths       the wavefront stages of ff_render (ff_wavefront.cu) in
//                     cache mode: a path ends at its first rough vertex after
//                     the camera hit with a query record; the cache's answers
//                     (throughput x max(cache, 0)) join the path sums before
//                     the film update.
// Record counts stay on the device.
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
    const FFTangentTri* tan;
    const ff_material* mats;
    const FFTexView* tex;
    const ff_area_light* area;
    FFEnvView env;
    FFLightSet lights;
    ff_camera cam;
    uint32_t W, H, frame, seed, max_depth, rr_depth, n_train;
    int32_t light;
    float shadow_offset, rough_threshold;
    Record* train;
    uint32_t* n_train_out;
    unsigned long long* rays;     // [0] extension, [1] shadow
    unsigned int* err;
};

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

using ffc::make_record;

__global__ void __launch_bounds__(kBlock) k_training_paths(CR a)
{
    __shared__ uint2 s_stack[kShortStack * kBlock];
    FFStack st;
    st.sm = s_stack + threadIdx.x;
    st.stride = kBlock;
    st.sp = 0;
    st.overflow = false;
    const uint32_t npix = a.W * a.H;
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = j < a.n_train;
    uint64_t n_ext = 0, n_shadow = 0;
    bool want_train = false;
    Record rec;
    if (active) {
        // a random pixel, samples independent of the frame's pixel paths
        const uint32_t h = ff_wang_hash(ff_wang_hash(a.seed ^ 0x6A09E667u) ^ ff_wang_hash(a.frame * 0x9E3779B9u + j));
        const uint32_t pix = (uint32_t)(((uint64_t)h * npix) >> 32);
        const uint32_t key = ff_path_key(a.seed ^ 0xBB67AE85u, pix, a.frame * a.n_train + j);
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
        bool inside = false;   // the ray runs inside an object: traced two-sided
        uint32_t L = 0;
        for (;;) {
            ff_hit hit;
            const bool found = ff_closest_hit(a.bvh, o, d, st, a.err, hit, inside);
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
            const float2 tuv = make_float2(u * t.uv1.x + v * t.uv2.x + wuv * t.uv0.x,
                                           u * t.uv1.y + v * t.uv2.y + wuv * t.uv0.y);
            const ff_material& mm = a.mats[t.material];
            float3 n = shading_normal(mm, a.tex, a.tan, prim, u, v, tuv, ng);
            if (back) {
                ng = -ng;
                n = -n;
            }
            const FFSurf surf = resolve_surface(mm, a.tex, tuv);
            const float3 wo = -d;
            if (L >= 2 && !tail && is_rough(surf, a.rough_threshold)) {
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
                case FF_MAT_MIX: shade_mix<true>(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, sp, key, L, sh); break;
                case FF_MAT_DIFFUSE: shade_diffuse<true>(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
                case FF_MAT_CONDUCTOR: shade_conductor<true>(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
                case FF_MAT_DIELECTRIC:
                    shade_dielectric(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, back, sh);
                    break;
                default: shade_coat(FF_MODE_CORRECTED, lc, surf, pos, n, wo, wi, key, L, sh); break;
            }
            const bool diel = surf.kind == FF_MAT_DIELECTRIC;
            const float3 lo = pos + ng * (((diel && dot3(wi, ng) < 0.f) ? -1.f : 1.f) * a.shadow_offset);
            sh.ray_nee = light_vis_ray(lc, lo, wi, key, L, DIM_NEE_VIS, sh.r_nee);
            vis = sh.ray_nee && !ff_occluded(a.bvh, sh.r_nee, st, a.err);
            vis_s = sh.ray_spec && !ff_occluded(a.bvh, sh.r_spec, st, a.err);
            vis_d = sh.ray_diff && !ff_occluded(a.bvh, sh.r_diff, st, a.err);
            n_shadow += (sh.ray_nee ? 1 : 0) + (sh.ray_spec ? 1 : 0) + (sh.ray_diff ? 1 : 0);
            const float side = dot3(sh.ext_d, ng) >= 0.f ? 1.f : -1.f;
            o = pos + ng * (side * a.shadow_offset);
            d = sh.ext_d;
            inside = runs_inside(back, diel, side);
        }
        if (want_train) {
            rec.v0 = Ltail.x;
            rec.v1 = Ltail.y;
            rec.v2 = Ltail.z;
            want_train = isfinite(Ltail.x) && isfinite(Ltail.y) && isfinite(Ltail.z);
        }
    }
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

__global__ void k_tally(const uint32_t* __restrict__ n, unsigned long long* __restrict__ total)
{
    total[0] += n[0];
    total[1] += n[1];
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
    a.tan = scene->tangent.as<FFTangentTri>();
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
    a.train = c->train_recs.as<Record>();
    a.n_train_out = cnt + 1;
    a.rays = rays;
    a.err = err;
    // the pixel paths: one sample per pixel per frame through the wavefront
    ff_render_settings ps = *st;
    ps.spp = 1;
    ps.mode = FF_MODE_CORRECTED;
    ps.max_paths = npix;
    ps.flags = 0;
    FFCacheHook hook{c, c->queries.ptr, cnt, npix, c->prm.rough_threshold, nullptr, nullptr, nullptr};
    const bool profile = (st->flags & FF_RENDER_PROFILE) != 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    for (auto& e : ev) FF_CUDA_CHECK(cudaEventCreate(&e));
    float ms_paths = 0.f, ms_train = 0.f;
    uint64_t launches = 0, ext = 0, shadow = 0;
    FF_CUDA_CHECK(cudaEventRecord(ev[0], stream));
    cudaEvent_t evq[2] = {nullptr, nullptr};
    if (profile) {
        for (auto& e : evq) FF_CUDA_CHECK(cudaEventCreate(&e));
        hook.ev_query0 = evq[0];
        hook.ev_query1 = evq[1];
    }
    float ms_query = 0.f;
    // Per frame, the training paths and the optimiser steps run on the
    // cache's own stream beside the pixel paths; the inference waits for
    // them, and the next frame's training waits for this frame's inference
    // (it reads the weights the training updates).
    cudaStream_t aux = c->aux;
    hook.wait_before_query = c->ev_trained;
    for (uint32_t f = 0; f < st->spp; ++f) {
        a.frame = st->sample_offset + f;
        FF_CUDA_CHECK(cudaEventRecord(c->ev_frame, stream));
        FF_CUDA_CHECK(cudaStreamWaitEvent(aux, c->ev_frame, 0));
        FF_CUDA_CHECK(cudaMemsetAsync(cnt + 1, 0, 4, aux));
        if (profile) FF_CUDA_CHECK(cudaEventRecord(ev[1], aux));
        if (n_train) {
            k_training_paths<<<(n_train + kBlock - 1) / kBlock, kBlock, 0, aux>>>(a);
            launches += 1;
        }
        for (uint32_t off = 0; off < n_train; off += batch) {
            ff_cache_launch_train_slice(c, a.train, off, std::min(batch, n_train - off), cnt + 1, aux);
            launches += 3;
        }
        if (profile) FF_CUDA_CHECK(cudaEventRecord(ev[2], aux));
        FF_CUDA_CHECK(cudaEventRecord(c->ev_trained, aux));
        ps.sample_offset = st->sample_offset + f;
        ff_render_stats ws{};
        ff_wavefront_render(ctx, scene, &ps, film, &ws, &hook);
        k_tally<<<1, 1, 0, stream>>>(cnt, totals);
        FF_CUDA_CHECK(cudaGetLastError());
        launches += ws.kernel_launches + 2;
        ext += ws.extension_rays;
        shadow += ws.shadow_rays;
        if (profile) {
            float t = 0.f;
            FF_CUDA_CHECK(cudaEventSynchronize(ev[2]));
            cudaEventElapsedTime(&t, ev[1], ev[2]);
            ms_train += t;
            cudaEventElapsedTime(&t, evq[0], evq[1]);
            ms_query += t;
            ms_paths += ws.ms_total - t;
        }
    }
    FF_CUDA_CHECK(cudaEventRecord(ev[3], stream));   // the last inference waited for the last training
    unsigned long long h[6] = {0, 0, 0, 0, 0, 0};
    FF_CUDA_CHECK(cudaMemcpyAsync(h, c->counters.as<char>() + 16, sizeof(h), cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaStreamSynchronize(stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[3]);
    for (auto& e : ev) cudaEventDestroy(e);
    for (auto& e : evq)
        if (e) cudaEventDestroy(e);
    if ((unsigned int)h[2]) throw FFError{FF_ERR_INTERNAL, "traversal exceeded its step bound (malformed BVH)"};
    if (stats) {
        stats->extension_rays = h[0] + ext;
        stats->shadow_rays = h[1] + shadow;
        stats->samples = (uint64_t)npix * st->spp;
        stats->frames = st->spp;
        stats->ms_total = ms;
        stats->kernel_launches = (uint32_t)launches;
        stats->ms_cache_paths = ms_paths;   // pixel paths (wavefront stages)
        stats->ms_cache_train = ms_train;   // training paths and optimiser steps
        stats->ms_cache_query = ms_query;   // k_cache_infer over the frame's queries
        stats->cache_queries = h[4];
        stats->cache_records = h[5];
    }
}
