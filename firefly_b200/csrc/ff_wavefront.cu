// ff_wavefront.cu — the wavefront path tracer behind ff_render.
//
// Replaces wavefront_pathtrace and its stages (CUDA-RayTracer/kernel.cu:
// wf_logic :298-455, wf_generate :458-485, wf_extend :488-523, wf_shadow
// :526-543, wf_mat_diffuse :546-577, wf_mat_cook :580-614, wf_mat_mix
// :617-651, driver :658-676) and the PathTracer frame loop
// (PathTracer.cpp:59-79).
//
// One frame advances every path in flight by one bounce, as in the
// reference:
//   k_logic    consume the previous extension hit and shadow answers; add
//              the NEE contribution, update the throughput, Russian roulette;
//              terminated paths start their next sample with a camera ray
//              (wf_generate fused in); continuing paths sample the light and
//              are compacted into one queue per material kind with warp
//              ballots.
//   k_shade<K> per material kind: BRDF_L / BRDF_f / BRDF_pdf of the
//              reference's mix material (or the single-lobe and added kinds),
//              the continuation ray, and up to three shadow rays: the NEE ray
//              of wf_shadow and the two BSDF-sampled visibility rays that
//              BRDF_L traces inline in the reference.
//   k_trace    closest-hit over the extension queue, any-hit over the shadow
//              queue (persistent kernel of ff_trace.cu, queue length read on
//              the device).
// The path pool has m slots per pixel; slot j always renders pixel j % (w*h)
// and samples j / (w*h) + k*m, and keeps a compensated (Kahan) FP32 sum of its
// radiance.  The film adds the m slot sums per pixel in a fixed order, so
// results do not depend on scheduling.  Frames repeat until no slot has work.
//
// The same stages run the path-replay adjoint (ff_render_adjoint): in the
// adjoint instantiations (k_logic<true>, k_shade<K, false, true>) each slot
// traces a sample once as the primal pass, keeps the sample's radiance L_s,
// then replays the same sample from its seed.  During the replay k_shade
// leaves each vertex's derivative terms in the slot, and k_logic, once the
// vertex's shadow rays are answered, scatters dL/d(texel) of the albedo
// texture, the roughness texture and the environment map.  The primal
// instantiations compile none of that code.
#include <algorithm>
#include <cstddef>
#include <vector>

#include "ff_adjoint.cuh"
#include "ff_internal.h"
#include "ff_paths.cuh"

namespace {

using namespace ffp;
using namespace ffadj;
constexpr int kKinds = 5;
// PH_DRAINED (deferred mode): finished, and the last pending light terms
// added, so later frames skip the slot without reading its records.
constexpr uint32_t PH_START = 0, PH_FLIGHT = 1, PH_DONE = 2, PH_DRAINED = 3;

// Path-pool size when ff_render_settings.max_paths is 0: m slots per pixel,
// m = min(spp, this / (w*h)), at least 1.  Measured on the 1.3M-triangle
// 1080p scene at 64 spp: 2M slots 419 ms, 4M 360 ms, 8M 347 ms, 16M 342 ms
// per step (bigger queues hide the traversal's latency better and need
// fewer frames); 8M slots hold about 3.6 GB of path state.
constexpr uint64_t kDefaultPoolTarget = 1ull << 23;

// Counter words of one frame (zeroed at the start of each frame); one block
// of kCtrStride words per frame parity.
enum { C_EXT = 0, C_SH = 1, C_MAT = 2, C_ACTIVE = 2 + kKinds, C_WORDS = 8 + kKinds };
constexpr uint32_t kCtrStride = 32;

// The slot's ray (origin, direction) and its visibility word: byte k = the
// any-hit trace's answer for shadow ray k (1 occluded), byte 3 = which shadow
// rays k_shade queued (bit k).
struct __align__(32) SlotRay {
    float ox, oy, oz;
    uint32_t vis;
    float dx, dy, dz, pad;
};
// What a vertex's shading leaves for k_logic.
struct __align__(32) SlotShade {
    float nee_x, nee_y, nee_z, pdf;   // c_nee, ext_pdf
    float f_x, f_y, f_z, cosine;      // ext_f, ext_cos
};
struct __align__(32) SlotMis {
    float spec_x, spec_y, spec_z, pad0;   // c_spec
    float diff_x, diff_y, diff_z, pad1;   // c_diff
};
// The vertex k_logic hands to k_shade.  word = material index (bits 0-23) |
// path length (bits 24-30) | hit from inside an object (bit 31).
struct __align__(32) SlotVtx {
    float px, py, pz;
    uint32_t word;
    float nx, ny, nz;   // shading normal
    uint32_t key;
    float wix, wiy, wiz;   // NEE direction
    float u;
    float wox, woy, woz;   // toward the previous vertex
    float v;
};
// Deferred light terms (ff_render without the cache): what a vertex's
// shading leaves for the k_logic two frames later, after the any-hit trace
// that runs beside the next frame has answered its shadow rays: the
// throughput at the vertex, the frame stamp, the three light terms and the
// rays queued.  Indexed [frame parity][slot].
struct __align__(32) SlotPend {
    float bx, by, bz;
    uint32_t stamp;   // frame + kStampBase of the shading; any other value: nothing pending
    float nee_x, nee_y, nee_z;
    uint32_t queued;  // bit k: shadow ray k was queued
    float spec_x, spec_y, spec_z, pad0;
    float diff_x, diff_y, diff_z, pad1;
};
static_assert(sizeof(SlotRay) == 32 && sizeof(SlotShade) == 32 && sizeof(SlotMis) == 32 && sizeof(SlotVtx) == 64 &&
                  sizeof(SlotPend) == 64,
              "slot records are whole 32-byte sectors");
constexpr uint32_t kStampBase = 16;
// Deferred mode: blocks per SM of the any-hit trace (its persistent grid, of
// 8 that fit), leaving the rest of each SM to k_logic and k_shade of the next
// frame.  Measured on the 1.3M-triangle scene at 64 spp: 3 blocks 262.7 ms
// per step, 4: 265.4-266.0, 5: 268.7, 6: 272.7; later, against 256.3-256.4
// with 3: 2 blocks 267.4-267.6, 1: 298.2 (the trace then outlasts the next
// frame, whose successor waits for it).
constexpr int kDeferShadowBlocks = 3;   // stamps of real frames are >= 16; 0 marks an empty record
constexpr uint32_t kVtxMatBits = 24, kVtxLenShift = 24, kVtxLenMask = 0x7f;
// Byte of shadow ray k's answer for slot s in the SlotRay array (the tag the
// any-hit trace writes to): the low three bytes of the vis word.
__device__ __forceinline__ uint32_t vis_byte(uint32_t s, uint32_t k)
{
    return (uint32_t)sizeof(SlotRay) * s + (uint32_t)offsetof(SlotRay, vis) + k;
}

struct WF {
    // launch constants
    uint32_t P, WH, W, H, m;
    uint32_t seed, max_depth, rr_depth, mode;
    int32_t light;
    float shadow_offset;
    // slot state
    uint32_t* samples_left;
    uint32_t* next_sample;
    uint32_t* key;
    uint32_t* length;
    uint32_t* phase;
    float4* beta;
    // Per-slot records that k_shade reaches through its material queue, i.e.
    // scattered over the slots: each is whole 32-byte sectors, so a scattered
    // access moves no bytes it does not use (a lone 16-byte field fetches or
    // fills a half-used sector).
    SlotRay* ray;     // the slot's current ray and its visibility word
    SlotShade* shd;   // k_shade -> k_logic: NEE term, continuation f / pdf / cos
    SlotMis* mis;     // k_shade -> k_logic: BSDF-sampled light terms (mix, dielectric)
    SlotVtx* vtx;     // k_logic -> k_shade: the vertex to shade
    float4* hit_ngeo;     // interpolated normal, written only under a normal texture
    float4* acc;
    float4* acc_c;
    uint32_t* cnt;
    // deferred light terms (defer = 1): the frame's parity and number, the
    // pending records and the any-hit answers (byte k of a slot's word: shadow
    // ray k occluded), both [2][P]; the shadow queue and the frame counters
    // are per parity too, so that the any-hit trace of frame f runs beside
    // k_logic and k_shade of frame f + 1
    uint32_t defer, par, frame;
    SlotPend* pend;
    uint32_t* vis2;
    // queues
    ff_ray* ext_rays;
    uint32_t* ext_tag;   // per queued extension ray: its slot
    ff_hit* ext_hits;    // per slot: the closest hit of its extension ray (written by k_trace)
    ff_ray* sh_rays;
    uint32_t* sh_tag;    // per queued shadow ray: the byte of its answer (vis_byte, or 4 * slot + k in vis2)
    uint32_t* mat_queue;   // kKinds * P
    uint32_t* ctr;         // C_WORDS
    unsigned long long* totals;  // [0] extension rays, [1] shadow rays, [2] samples
    // scene
    const FFShadeTri* shade;
    const FFTangentTri* tan;   // tangent frames, or null when no material has a normal texture
    const ff_material* mats;
    const ff_area_light* area;
    uint32_t n_area;
    const FFTexView* tex;
    FFEnvView env;
    FFLightSet lights;
    ff_camera cam;
    // learned radiance cache (ff_render_cached): a path ends at its first
    // rough vertex after the camera hit and leaves a query record there
    uint32_t cache_mode;
    float rough_threshold;
    ffc::Record* queries;
    uint32_t* n_queries;
    // path-replay adjoint (null / -1 in ff_render)
    const float* d_image;        // W*H*3: dL/dI of the mean-radiance image
    float inv_spp;
    int32_t adj_texture;         // albedo texture receiving gradients, -1 none
    float* grad_tex;
    float* grad_env;             // null: no environment gradient
    int32_t adj_rough;           // roughness texture receiving gradients, -1 none
    float* grad_rough;           // null: no roughness gradient
    unsigned long long* touched; // [0] albedo/env texel touches, [1] roughness texel touches
    uint32_t* pass;              // per slot: 0 primal pass, 1 replay
    float4* l_total;             // per slot: L_s of the sample being replayed
    float4* v_albedo;            // per slot, last vertex: albedo, w = V_* flag bits
    float4* v_nee;               // d c_nee / dr
    float4* v_spec;              // d c_spec / dr
    float4* v_dext;              // d log(ext_f) / dr
    float4* v_coef;              // c_nee / Le(wi): d c_nee / d Le
};
// flags of WF::v_albedo.w: which gradients the vertex takes
constexpr uint32_t V_ALBEDO = 1u, V_ROUGH = 2u, V_ENV = 4u, V_ROUGH_Y = 8u;   // V_ROUGH_Y: roughness in channel y

__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 f4(float3 v, float w = 0.f) { return make_float4(v.x, v.y, v.z, w); }

// Warp-aggregated append (the reference's atomicAggInc, kernel.cu:24-36, on
// *_sync intrinsics): one atomic per warp and per queue.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want, unsigned long long* total)
{
    const uint32_t mask = __ballot_sync(__activemask(), want);
    if (!want) return 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) {
        base = atomicAdd(counter, (uint32_t)__popc(mask));
        if (total) atomicAdd(total, (unsigned long long)__popc(mask));
    }
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ void kahan_add(float4& sum, float4& c, float3 x)
{
    float3 y = make_float3(x.x - c.x, x.y - c.y, x.z - c.z);
    float3 t = make_float3(sum.x + y.x, sum.y + y.y, sum.z + y.z);
    c = make_float4((t.x - sum.x) - y.x, (t.y - sum.y) - y.y, (t.z - sum.z) - y.z, 0.f);
    sum = make_float4(t.x, t.y, t.z, 0.f);
}

__device__ __forceinline__ uint32_t slot_pixel(const WF& w, uint32_t s) { return s % w.WH; }

// wf_generate + dCamera::gen_ray for slot s, sample `sample`.
__device__ void start_sample(const WF& w, uint32_t s, uint32_t sample, bool& push, ff_ray& ray)
{
    const uint32_t pix = slot_pixel(w, s);
    const uint32_t key = ff_path_key(w.seed, pix, sample);
    w.key[s] = key;
    w.length[s] = 0;
    w.beta[s] = make_float4(1.f, 1.f, 1.f, 0.f);
    const int x = (int)(pix % w.W), y = (int)(pix / w.W);
    float3 o, d;
    gen_camera_ray(w.cam, (int)w.W, (int)w.H, x, y, rand2(key, 0, DIM_CAM_JITTER), rand2(key, 0, DIM_CAM_LENS), o, d);
    w.ray[s] = SlotRay{o.x, o.y, o.z, 0u, d.x, d.y, d.z, 0.f};
    ray = ff_ray{o.x, o.y, o.z, 0.f, d.x, d.y, d.z, __int_as_float(0x7f800000)};
    push = true;
}

// Deferred mode: the light terms of the vertex slot s shaded two frames ago
// (its pending record of this frame's parity, stamp frame - 2), gated by
// their shadow rays' answers exactly as k_logic gates them without
// deferral, into the slot's compensated sum.  Returns whether anything was
// pending.
__device__ __forceinline__ bool consume_pending(const WF& w, uint32_t s, float4& acc, float4& accc)
{
    const size_t i = (size_t)w.par * w.P + s;
    const float4* pq = reinterpret_cast<const float4*>(w.pend + i);
    const float4 a = pq[0];
    if (__float_as_uint(a.w) != w.frame + kStampBase - 2u) return false;
    const float4 b = pq[1];
    const uint32_t q = __float_as_uint(b.w);
    const uint32_t vw = w.vis2[i];
    const bool vis = (q & 1u) && !(vw & 0xffu);
    const bool vis_s = (q & 2u) && !(vw & 0xff00u);
    const bool vis_d = (q & 4u) && !(vw & 0xff0000u);
    const float3 beta = xyz(a);
    if (w.mode == FF_MODE_CORRECTED) {
        float3 lb = make_float3(0.f, 0.f, 0.f);
        if (vis) lb = lb + xyz(b);
        if (vis_s) lb = lb + xyz(pq[2]);
        if (vis_d) lb = lb + xyz(pq[3]);
        if (vis || vis_s || vis_d) kahan_add(acc, accc, lb * beta);
    } else if (vis) {
        // parity: the whole light_brdf, MIS terms included, rides on the NEE ray
        float3 lb = xyz(b);
        if (vis_s) lb = lb + xyz(pq[2]);
        if (vis_d) lb = lb + xyz(pq[3]);
        kahan_add(acc, accc, lb * beta);
    }
    return true;
}

// ADJ: the path-replay adjoint's instantiation (the slot's sum holds the
// current sample's radiance only, in plain FP32 adds as the megakernel
// adjoint sums it; no film).
template <bool ADJ>
__global__ void __launch_bounds__(256) k_logic(WF w)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    bool push_ext = false;
    ff_ray ray{};
    int kind = -1;
    bool active = false;
    uint32_t touched = 0, touched_r = 0;
    if (s < w.P) {
        uint32_t ph = w.phase[s];
        if (ph == PH_START) {
            const uint32_t smp = w.next_sample[s];
            w.next_sample[s] = smp + w.m;
            start_sample(w, s, smp, push_ext, ray);
            w.phase[s] = PH_FLIGHT;
            if (ADJ) {
                w.pass[s] = 0;
                w.acc[s] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            active = true;
        } else if (ph == PH_FLIGHT) {
            active = true;
            const uint32_t key = w.key[s];
            const ff_hit hit = w.ext_hits[s];
            const uint32_t L = w.length[s] + 1;  // wf_extend's length++
            const bool found = hit.prim != -1;
            const SlotRay sr = w.ray[s];
            const float3 ro = make_float3(sr.ox, sr.oy, sr.oz), rd = make_float3(sr.dx, sr.dy, sr.dz);
            float3 beta = xyz(w.beta[s]);
            float4 acc = w.acc[s];
            float4 accc = ADJ ? make_float4(0.f, 0.f, 0.f, 0.f) : w.acc_c[s];   // no compensation in the adjoint
            if (!ADJ && w.defer) consume_pending(w, s, acc, accc);
            bool terminate = (L > w.max_depth) || !found;
            // adjoint replay: dL/dI of this sample's pixel and the primal pass's L_s
            const bool replay = ADJ && w.pass[s] != 0u;
            float3 dI = make_float3(0.f, 0.f, 0.f), Ltot = make_float3(0.f, 0.f, 0.f);
            if (replay) {
                const uint32_t pix = slot_pixel(w, s);
                dI = make_float3(w.d_image[3 * (size_t)pix] * w.inv_spp, w.d_image[3 * (size_t)pix + 1] * w.inv_spp,
                                 w.d_image[3 * (size_t)pix + 2] * w.inv_spp);
                Ltot = xyz(w.l_total[s]);
            }
            // kernel.cu:332-338: environment radiance on a camera-ray miss
            if (!found && L == 1) {
                if (ADJ) {
                    const float3 c = beta * env_L(w.env, rd, true);
                    if (replay && w.grad_env && w.env.rgb) {
                        float3 dd = rd;
                        dd.y = clampf(dd.y, -1.f, 1.f);
                        const float2 euv = spherical_map(dd);
                        touched += scatter_footprint(w.grad_env, footprint(w.env.width, w.env.height, euv.x, euv.y),
                                                     dI * beta);
                    }
                    acc = f4(xyz(acc) + c);
                } else {
                    kahan_add(acc, accc, beta * env_L(w.env, rd, w.mode == FF_MODE_CORRECTED));
                }
            }
            if (L > 1) {
                const SlotShade sd = w.shd[s];
                if (ADJ || !w.defer) {   // (deferred light terms were added above)
                    // kernel.cu:357-359: light_brdf * beta when the NEE ray was unoccluded
                    const uint32_t vw = sr.vis;
                    const bool vis = (vw & (1u << 24)) && !(vw & 0xffu);
                    const bool vis_s = (vw & (2u << 24)) && !(vw & 0xff00u);
                    const bool vis_d = (vw & (4u << 24)) && !(vw & 0xff0000u);
                    if (w.mode == FF_MODE_CORRECTED) {
                        // every term gated by its own visibility ray
                        float3 lb = make_float3(0.f, 0.f, 0.f);
                        if (vis) lb = lb + make_float3(sd.nee_x, sd.nee_y, sd.nee_z);
                        if (vis_s || vis_d) {
                            const SlotMis sm = w.mis[s];
                            if (vis_s) lb = lb + make_float3(sm.spec_x, sm.spec_y, sm.spec_z);
                            if (vis_d) lb = lb + make_float3(sm.diff_x, sm.diff_y, sm.diff_z);
                        }
                        if (ADJ) {
                            if (replay) {
                                // the previous vertex's gradients, now that its shadow rays are answered
                                const float4 va = w.v_albedo[s];
                                const uint32_t flags = __float_as_uint(va.w);
                                const SlotVtx& pv = w.vtx[s];   // the previous vertex
                                const float2 uv = make_float2(pv.u, pv.v);
                                if (flags & V_ALBEDO) {
                                    const FFTexView tv = w.tex[w.adj_texture];
                                    touched += scatter_footprint(w.grad_tex, footprint(tv.width, tv.height, uv.x, uv.y),
                                                                 albedo_grad(Ltot - xyz(acc), xyz(va), dI));
                                }
                                if (flags & V_ROUGH) {
                                    RoughTerms rt;
                                    rt.nee = xyz(w.v_nee[s]);
                                    rt.spec = xyz(w.v_spec[s]);
                                    rt.dext = xyz(w.v_dext[s]);
                                    const float3 rimm = rough_own(rt, vis, vis_s, beta);
                                    const float3 L_after = xyz(acc) + lb * beta;
                                    const float g = dot3(dI, rimm + (Ltot - L_after) * rt.dext);
                                    const FFTexView tv = w.tex[w.adj_rough];
                                    touched_r += scatter_footprint1(w.grad_rough, footprint(tv.width, tv.height, uv.x, uv.y), g,
                                                                    (flags & V_ROUGH_Y) ? 1 : 0);
                                }
                                if ((flags & V_ENV) && vis) {
                                    // NEE term c_nee = coef * Le(wi): d/dLe = beta * coef
                                    float3 wl = make_float3(pv.wix, pv.wiy, pv.wiz);
                                    wl.y = clampf(wl.y, -1.f, 1.f);
                                    const float2 euv = spherical_map(wl);
                                    touched += scatter_footprint(w.grad_env, footprint(w.env.width, w.env.height, euv.x, euv.y),
                                                                 dI * beta * xyz(w.v_coef[s]));
                                }
                            }
                            if (vis || vis_s || vis_d) acc = f4(xyz(acc) + lb * beta);
                        } else if (vis || vis_s || vis_d) {
                            kahan_add(acc, accc, lb * beta);
                        }
                    } else if (!ADJ && vis) {
                        // parity: the whole light_brdf, MIS terms included, rides on the NEE ray
                        float3 lb = make_float3(sd.nee_x, sd.nee_y, sd.nee_z);
                        if (vis_s || vis_d) {
                            const SlotMis sm = w.mis[s];
                            if (vis_s) lb = lb + make_float3(sm.spec_x, sm.spec_y, sm.spec_z);
                            if (vis_d) lb = lb + make_float3(sm.diff_x, sm.diff_y, sm.diff_z);
                        }
                        kahan_add(acc, accc, lb * beta);
                    }
                }
                const float3 f = make_float3(sd.f_x, sd.f_y, sd.f_z);
                const float pdf = sd.pdf;
                const float cosine = sd.cosine;
                if (f == make_float3(0.f, 0.f, 0.f) || pdf == 0.f) {
                    terminate = true;
                } else {
                    beta *= (f * cosine) / pdf;
                    if (L > w.rr_depth) {
                        const float q_rr = hmax(0.05f, 1.f - beta.y);
                        if (ff_rand(key, dim_of(L, DIM_RR)) < q_rr) terminate = true;
                        else if (w.mode == FF_MODE_CORRECTED) {
                            // a draw of exactly 1.0 survives q = 1: no finite compensation exists
                            if (q_rr >= 1.f) terminate = true;
                            else beta = beta / (1.f - q_rr);
                        }
                    }
                }
            }
            w.acc[s] = acc;
            if (!ADJ) w.acc_c[s] = accc;
            bool query = false;
            ffc::Record rec;
            if (!terminate) {
                // Continue: hit attributes (dTriangle::hit, dTriangle.cu:94-105).
                const bool back = hit_back(hit.prim);
                const uint32_t prim = hit_index(hit.prim);
                const FFShadeRec t = ff_load_shade(w.shade, prim);
                const float u = hit.u, v = hit.v;
                float3 n = normalize3(u * t.n1 + v * t.n2 + ((1.f - u) - v) * t.n0);
                const float3 pos = ro + hit.t * rd;
                // texcoord = u * uv1 + v * uv2 + (1 - u - v) * uv0 (dTriangle.cu:97)
                const float wuv = (1.f - u) - v;
                const float2 uv = make_float2(u * t.uv1.x + v * t.uv2.x + wuv * t.uv0.x,
                                              u * t.uv1.y + v * t.uv2.y + wuv * t.uv0.y);
                const ff_material& mm = w.mats[t.material];
                // get_normal: the shading normal (a normal texture's frame, else
                // n); n stays the normal the ray offsets follow (kernel.cu:437)
                float3 ns = shading_normal(mm, w.tex, w.tan, prim, u, v, uv, n);
                if (back) {   // a back face of a two-sided ray: shaded from the inside
                    n = -n;
                    ns = -ns;
                }
                if (!ADJ && w.cache_mode && L >= 2) {
                    const FFSurf surf = resolve_surface(mm, w.tex, uv);
                    if (is_rough(surf, w.rough_threshold)) {
                        // the cache answers for everything from this vertex on
                        rec = ffc::make_record(pos, surf.roughness, -rd, ns, beta, s);
                        query = true;
                        terminate = true;
                    }
                }
                if (!query) {
                    // Light sample (kernel.cu:435, light get_direction).
                    float3 wi, sp;
                    sample_light(select_light(w.lights, key, L), pos, key, L, wi, sp);
                    w.length[s] = L;
                    w.beta[s] = f4(beta);
                    SlotVtx vx;
                    vx.px = pos.x, vx.py = pos.y, vx.pz = pos.z;
                    vx.word = t.material | (L << kVtxLenShift) | (back ? kBackFace : 0u);
                    vx.nx = ns.x, vx.ny = ns.y, vx.nz = ns.z;
                    vx.key = key;
                    vx.wix = wi.x, vx.wiy = wi.y, vx.wiz = wi.z;   // (the sample point is not needed downstream)
                    vx.u = uv.x;
                    vx.wox = -rd.x, vx.woy = -rd.y, vx.woz = -rd.z;
                    vx.v = uv.y;
                    w.vtx[s] = vx;
                    if (mm.normal_tex >= 0) w.hit_ngeo[s] = f4(n);
                    kind = mm.kind;
                }
            }
            if (terminate) {
                if (ADJ && !replay) {
                    // primal pass done: keep L_s and replay the same sample from its seed
                    w.l_total[s] = acc;
                    w.pass[s] = 1u;
                    w.acc[s] = make_float4(0.f, 0.f, 0.f, 0.f);
                    start_sample(w, s, w.next_sample[s] - w.m, push_ext, ray);
                } else {
                    w.cnt[s] += 1u;
                    const uint32_t left = w.samples_left[s] - 1u;
                    w.samples_left[s] = left;
                    if (ADJ) {
                        w.pass[s] = 0u;
                        w.acc[s] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                    if (left > 0) {
                        const uint32_t smp = w.next_sample[s];
                        w.next_sample[s] = smp + w.m;
                        start_sample(w, s, smp, push_ext, ray);
                    } else {
                        w.phase[s] = PH_DONE;
                        active = false;
                    }
                }
            }
            if (!ADJ && w.cache_mode) {
                const uint32_t qi = warp_append(w.n_queries, query, nullptr);
                if (query) w.queries[qi] = rec;
            }
        } else if (!ADJ && w.defer && ph == PH_DONE) {
            // a slot that finished in the previous frame: the light terms of its
            // last vertex (shaded two frames ago) are the only ones still pending
            float4 acc = w.acc[s], accc = w.acc_c[s];
            if (consume_pending(w, s, acc, accc)) {
                w.acc[s] = acc;
                w.acc_c[s] = accc;
            }
            w.phase[s] = PH_DRAINED;
        }
    }
    // compaction into the extension queue and the material queues
    const uint32_t qe = warp_append(&w.ctr[C_EXT], push_ext, &w.totals[0]);
    if (push_ext) {
        w.ext_rays[qe] = ray;
        w.ext_tag[qe] = s;
    }
#pragma unroll
    for (int k = 0; k < kKinds; ++k) {
        const uint32_t qm = warp_append(&w.ctr[C_MAT + k], kind == k, nullptr);
        if (kind == k) w.mat_queue[(size_t)k * w.P + qm] = s;
    }
    const uint32_t am = __ballot_sync(0xffffffffu, active);
    if ((threadIdx.x & 31u) == 0 && am) atomicAdd(&w.ctr[C_ACTIVE], (uint32_t)__popc(am));
    if (ADJ) {
        touched = __reduce_add_sync(0xffffffffu, touched);
        touched_r = __reduce_add_sync(0xffffffffu, touched_r);
        if ((threadIdx.x & 31u) == 0) {
            if (touched) atomicAdd(&w.touched[0], (unsigned long long)touched);
            if (touched_r) atomicAdd(&w.touched[1], (unsigned long long)touched_r);
        }
    }
}

// SEL: the light is chosen per vertex (FF_LIGHT_ALL); otherwise one light
// context serves the whole launch (fewer live registers).  ADJ: the adjoint's
// instantiation, which also leaves the vertex's derivative terms in the slot
// during a replay.  CORR: corrected mode, whose reference lobes run in FP32
// (parity mode keeps the reference's FP64 arithmetic; Lobes, ff_shade.cuh).
template <int KIND, bool SEL, bool ADJ, bool CORR>
__global__ void __launch_bounds__(128) k_shade(WF w)
{
    const uint32_t n = w.ctr[C_MAT + KIND];
    const uint32_t stride = gridDim.x * blockDim.x;
    // every lane runs the same number of iterations so the queue appends can use full-warp ballots
    const uint32_t iters = (n + stride - 1) / stride;
    const uint32_t base = blockIdx.x * blockDim.x + threadIdx.x;
    LightCtx lc;
    if (!SEL) lc = select_light(w.lights, 0u, 0u);   // the fixed light
    for (uint32_t it = 0; it < iters; ++it) {
        const uint32_t qi = base + it * stride;
        const bool valid = qi < n;
        ShadeOut o;
        o.ray_nee = o.ray_spec = o.ray_diff = false;
        bool ext_two = false;   // the continuation runs inside an object: traced two-sided
        uint32_t s = 0;
        float4 beta_v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (valid) {
            s = w.mat_queue[(size_t)KIND * w.P + qi];
            const SlotVtx vx = w.vtx[s];
            const float3 pos = make_float3(vx.px, vx.py, vx.pz);
            const bool back = (vx.word & kBackFace) != 0;   // hit from inside an object
            const ff_material& mm = w.mats[vx.word & ((1u << kVtxMatBits) - 1u)];
            const FFSurf mat = resolve_surface(mm, w.tex, make_float2(vx.u, vx.v));
            const float3 n = make_float3(vx.nx, vx.ny, vx.nz);   // shading normal
            // the normal the ray offsets follow (kernel.cu:437): differs from n
            // only under a normal texture
            const float3 ng = mm.normal_tex >= 0 ? xyz(w.hit_ngeo[s]) : n;
            const float3 wo = make_float3(vx.wox, vx.woy, vx.woz);
            const float3 wi = make_float3(vx.wix, vx.wiy, vx.wiz);
            const float3 sp = make_float3(0.f, 0.f, 0.f);   // BRDF_L does not use the NEE sample point
            const uint32_t key = vx.key;
            const uint32_t L = (vx.word >> kVtxLenShift) & kVtxLenMask;
            if (SEL) lc = select_light(w.lights, key, L);
            o.c_spec = o.c_diff = make_float3(0.f, 0.f, 0.f);
            if (KIND == FF_MAT_MIX) shade_mix<CORR>(w.mode, lc, mat, pos, n, wo, wi, sp, key, L, o);
            else if (KIND == FF_MAT_DIFFUSE) shade_diffuse<CORR>(w.mode, lc, mat, pos, n, wo, wi, key, L, o);
            else if (KIND == FF_MAT_CONDUCTOR) shade_conductor<CORR>(w.mode, lc, mat, pos, n, wo, wi, key, L, o);
            else if (KIND == FF_MAT_DIELECTRIC) shade_dielectric(w.mode, lc, mat, pos, n, wo, wi, key, L, back, o);
            else shade_coat(w.mode, lc, mat, pos, n, wo, wi, key, L, o);
            // NEE shadow ray of wf_shadow: light_ray = position + normal * SHADOW_OFFSET (kernel.cu:437);
            // a dielectric's light may lie on the far side
            const float nee_side = (KIND == FF_MAT_DIELECTRIC && dot3(wi, ng) < 0.f) ? -1.f : 1.f;
            const float3 lo = pos + ng * (nee_side * w.shadow_offset);
            o.ray_nee = light_vis_ray(lc, lo, wi, key, L, DIM_NEE_VIS, o.r_nee);
            // continuation ray: the reference starts it at the hit point (kernel.cu:643);
            // corrected mode, and every ray that leaves a dielectric or an
            // inside vertex, starts off the surface on the side it leaves
            const float side = dot3(o.ext_d, ng) >= 0.f ? 1.f : -1.f;
            o.ext_o = pos;
            if (w.mode == FF_MODE_CORRECTED || KIND == FF_MAT_DIELECTRIC || back)
                o.ext_o = pos + ng * (side * w.shadow_offset);
            ext_two = runs_inside(back, KIND == FF_MAT_DIELECTRIC, side);
            w.shd[s] = SlotShade{o.c_nee.x, o.c_nee.y, o.c_nee.z, o.ext_pdf, o.ext_f.x, o.ext_f.y, o.ext_f.z, o.ext_cos};
            // the kinds with BSDF-sampled light terms (deferred mode: in the pending record)
            if ((KIND == FF_MAT_MIX || KIND == FF_MAT_DIELECTRIC) && (ADJ || !w.defer))
                w.mis[s] = SlotMis{o.c_spec.x, o.c_spec.y, o.c_spec.z, 0.f, o.c_diff.x, o.c_diff.y, o.c_diff.z, 0.f};
            if (ADJ && w.pass[s] != 0u) {
                uint32_t flags = 0;
                if (KIND == FF_MAT_DIFFUSE && w.grad_tex && mm.base_color_tex >= 0 && mm.base_color_tex == w.adj_texture)
                    flags |= V_ALBEDO;
                // roughness from the texture, above the 0.01 floor of resolve_surface (flat there)
                const int rch = KIND != FF_MAT_DIFFUSE && w.grad_rough ? rough_channel(mm, w.adj_rough) : -1;
                if (rch >= 0 && mat.roughness > 0.01f) {
                    flags |= V_ROUGH | (rch == 1 ? V_ROUGH_Y : 0u);
                    const RoughTerms rt = rough_terms(o, n, wo, wi, mat.roughness, KIND == FF_MAT_DIELECTRIC);
                    w.v_nee[s] = f4(rt.nee);
                    w.v_spec[s] = f4(rt.spec);
                    w.v_dext[s] = f4(rt.dext);
                }
                if (w.grad_env && lc.is_env && w.env.rgb) {
                    // c_nee is linear in Le(wi)
                    const float3 Li = light_L(lc, wi);
                    w.v_coef[s] = make_float4(Li.x != 0.f ? o.c_nee.x / Li.x : 0.f, Li.y != 0.f ? o.c_nee.y / Li.y : 0.f,
                                              Li.z != 0.f ? o.c_nee.z / Li.z : 0.f, 0.f);
                    flags |= V_ENV;
                }
                w.v_albedo[s] = f4(mat.albedo, __uint_as_float(flags));
            }
        }
        const uint32_t qe = warp_append(&w.ctr[C_EXT], valid, &w.totals[0]);
        if (valid) {
            w.ext_rays[qe] = make_ext_ray(o.ext_o, o.ext_d, ext_two);
            w.ext_tag[qe] = s;
        }
        const uint32_t q0 = warp_append(&w.ctr[C_SH], o.ray_nee, &w.totals[1]);
        const uint32_t q1 = warp_append(&w.ctr[C_SH], o.ray_spec, &w.totals[1]);
        const uint32_t q2 = warp_append(&w.ctr[C_SH], o.ray_diff, &w.totals[1]);
        // answer tags: bytes of the slot's vis word in SlotRay, or of its word in vis2 (deferred mode)
        const bool defer = !ADJ && w.defer;
        if (o.ray_nee) {
            w.sh_rays[q0] = o.r_nee;
            w.sh_tag[q0] = defer ? 4u * s : vis_byte(s, 0);
        }
        if (o.ray_spec) {
            w.sh_rays[q1] = o.r_spec;
            w.sh_tag[q1] = defer ? 4u * s + 1u : vis_byte(s, 1);
        }
        if (o.ray_diff) {
            w.sh_rays[q2] = o.r_diff;
            w.sh_tag[q2] = defer ? 4u * s + 2u : vis_byte(s, 2);
        }
        if (valid) {
            // the continuation ray and the queued-rays byte, one whole record
            const uint32_t queued = ((o.ray_nee ? 1u : 0u) | (o.ray_spec ? 2u : 0u) | (o.ray_diff ? 4u : 0u)) << 24;
            w.ray[s] = SlotRay{o.ext_o.x, o.ext_o.y, o.ext_o.z, queued, o.ext_d.x, o.ext_d.y, o.ext_d.z, 0.f};
            if (defer) {
                // the light terms with the throughput they multiply, for k_logic two frames on
                beta_v = w.beta[s];   // the throughput at this vertex
                float4* pq = reinterpret_cast<float4*>(w.pend + (size_t)w.par * w.P + s);
                pq[0] = make_float4(beta_v.x, beta_v.y, beta_v.z, __uint_as_float(w.frame + kStampBase));
                pq[1] = make_float4(o.c_nee.x, o.c_nee.y, o.c_nee.z, __uint_as_float(queued >> 24));
                pq[2] = f4(o.c_spec);
                pq[3] = f4(o.c_diff);
            }
        }
    }
}

__global__ void k_init(WF w, uint32_t spp, uint32_t sample_offset)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= w.P) return;
    if (w.pass) w.pass[s] = 0u;
    const uint32_t lane = s / w.WH;  // which of the m slots of its pixel
    const uint32_t left = lane < spp ? (spp - lane + w.m - 1) / w.m : 0u;
    w.samples_left[s] = left;
    w.next_sample[s] = sample_offset + lane;
    w.phase[s] = left ? PH_START : PH_DONE;
    w.acc[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    w.acc_c[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    w.cnt[s] = 0;
    w.ray[s].vis = 0u;
    if (w.defer) {
        w.pend[s].stamp = 0u;
        w.pend[(size_t)w.P + s].stamp = 0u;
    }
}

// Deferred mode: the light terms still pending after the last frame (stamp
// w.frame - 2 of the parity of w.frame).
__global__ void k_flush_pending(WF w)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= w.P) return;
    float4 acc = w.acc[s], accc = w.acc_c[s];
    if (consume_pending(w, s, acc, accc)) {
        w.acc[s] = acc;
        w.acc_c[s] = accc;
    }
}

// Film += the m slot sums of each pixel, in slot order (compensated).
__global__ void k_resolve(WF w, float4* __restrict__ film_acc, float4* __restrict__ film_c, uint32_t* __restrict__ film_n)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= w.WH) return;
    float4 sum = film_acc[p], c = film_c[p];
    uint32_t n = film_n[p];
    for (uint32_t k = 0; k < w.m; ++k) {
        const uint32_t s = p + k * w.WH;
        const float4 a = w.acc[s], ac = w.acc_c[s];
        kahan_add(sum, c, make_float3(a.x - ac.x, a.y - ac.y, a.z - ac.z));
        n += w.cnt[s];
    }
    film_acc[p] = sum;
    film_c[p] = c;
    film_n[p] = n;
}

__global__ void k_reset_counters(uint32_t* ctr, unsigned long long* trace_counters)
{
    if (threadIdx.x < C_WORDS) ctr[threadIdx.x] = 0;
    if (threadIdx.x < 2) trace_counters[threadIdx.x] = 0ull;
}

}  // namespace

// Per-film workspace: slot arrays and queues, reused while the pool size is unchanged.
struct FFWavefrontWS {
    uint32_t P = 0;
    DevBuf buf;
    DevBuf adj_buf;   // the adjoint's per-slot arrays (allocated by ff_wavefront_adjoint only)
    DevBuf defer_buf; // the deferred light terms' arrays (allocated by ff_render only)
    uint32_t defer_P = 0;
    uint32_t adj_P = 0;
    WF w{};
    unsigned int* err = nullptr;
    unsigned long long* trace_ctr = nullptr;  // per frame parity p: [2p] closest, [2p + 1] any
    // per frame parity p: the counter words (ctr_base + kCtrStride * p) and the
    // shadow queue (sh_rays_base[p], sh_tag_base[p]); WF points at the current
    // frame's
    uint32_t* ctr_base = nullptr;
    ff_ray* sh_rays_base[2] = {nullptr, nullptr};
    uint32_t* sh_tag_base[2] = {nullptr, nullptr};
    unsigned long long* fetch = nullptr;      // profiled renders: nodes / tris of the closest, then the any-hit traces
    uint32_t* h_active = nullptr;             // pinned host word for the frame-loop check
    // the any-hit trace runs on `side` beside the closest-hit trace: its
    // blocks take the SMs the closest-hit trace's finished blocks leave
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // deferred mode: the any-hit trace of the last frame of each parity done
    cudaEvent_t sh_done[2] = {nullptr, nullptr};
    // k_shade of the second to fifth material kind in use, beside the first
    cudaStream_t kind_side[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t kind_join[4] = {nullptr, nullptr, nullptr, nullptr};
    void ensure_streams()
    {
        if (side) return;
        FF_CUDA_CHECK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        FF_CUDA_CHECK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        FF_CUDA_CHECK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
        for (int i = 0; i < 2; ++i) FF_CUDA_CHECK(cudaEventCreateWithFlags(&sh_done[i], cudaEventDisableTiming));
        for (int i = 0; i < 4; ++i) {
            FF_CUDA_CHECK(cudaStreamCreateWithFlags(&kind_side[i], cudaStreamNonBlocking));
            FF_CUDA_CHECK(cudaEventCreateWithFlags(&kind_join[i], cudaEventDisableTiming));
        }
    }
    ~FFWavefrontWS()
    {
        if (h_active) cudaFreeHost(h_active);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        for (int i = 0; i < 2; ++i)
            if (sh_done[i]) cudaEventDestroy(sh_done[i]);
        if (side) cudaStreamDestroy(side);
        for (int i = 0; i < 4; ++i) {
            if (kind_join[i]) cudaEventDestroy(kind_join[i]);
            if (kind_side[i]) cudaStreamDestroy(kind_side[i]);
        }
    }
};

void ff_wavefront_ws_free(FFWavefrontWS* ws) { delete ws; }

namespace {

template <class T>
T* carve(char*& p, size_t n)
{
    T* r = reinterpret_cast<T*>(p);
    size_t bytes = (sizeof(T) * n + 255) & ~size_t(255);
    p += bytes;
    return r;
}

template <int K, bool SEL, bool ADJ, bool CORR>
void shade_kind(const WF& w, int blocks, cudaStream_t stream)
{
    k_shade<K, SEL, ADJ, CORR><<<blocks, 128, 0, stream>>>(w);
}

// k_shade for every material kind in use.  With ws, the first kind runs on
// `stream` and each further kind on a side stream of its own, all after the
// work already on `stream` (k_logic); `stream` then waits for all of them.
// The kinds shade disjoint slots and append to the queues with atomics, so
// the order of their launches does not change any result.
template <bool SEL, bool ADJ, bool CORR>
void launch_shade(const WF& w, const bool* kind_used, int blocks, cudaStream_t stream, FFWavefrontWS* ws)
{
    using Fn = void (*)(const WF&, int, cudaStream_t);
    Fn fns[kKinds];
    fns[FF_MAT_MIX] = shade_kind<FF_MAT_MIX, SEL, ADJ, CORR>;
    fns[FF_MAT_DIFFUSE] = shade_kind<FF_MAT_DIFFUSE, SEL, ADJ, CORR>;
    fns[FF_MAT_CONDUCTOR] = shade_kind<FF_MAT_CONDUCTOR, SEL, ADJ, CORR>;
    fns[FF_MAT_DIELECTRIC] = shade_kind<FF_MAT_DIELECTRIC, SEL, ADJ, CORR>;
    fns[FF_MAT_COAT] = shade_kind<FF_MAT_COAT, SEL, ADJ, CORR>;
    int n_side = 0;
    bool first = true;
    if (ws) FF_CUDA_CHECK(cudaEventRecord(ws->fork, stream));
    for (int k = 0; k < kKinds; ++k) {
        if (!kind_used[k]) continue;
        if (!ws || first) {
            fns[k](w, blocks, stream);
            first = false;
            continue;
        }
        cudaStream_t s = ws->kind_side[n_side];
        FF_CUDA_CHECK(cudaStreamWaitEvent(s, ws->fork, 0));
        fns[k](w, blocks, s);
        FF_CUDA_CHECK(cudaEventRecord(ws->kind_join[n_side], s));
        ++n_side;
    }
    for (int i = 0; i < n_side; ++i) FF_CUDA_CHECK(cudaStreamWaitEvent(stream, ws->kind_join[i], 0));
}

size_t ws_bytes(uint32_t P)
{
    size_t b = 0;
    auto add = [&](size_t s, size_t n) { b += (s * n + 255) & ~size_t(255); };
    add(4, P) /*samples_left*/; add(4, P); add(4, P); add(4, P); add(4, P);
    add(16, P) /*beta*/; add(sizeof(SlotRay), P); add(sizeof(SlotShade), P); add(sizeof(SlotMis), P);
    add(sizeof(SlotVtx), P); add(16, P) /*hit_ngeo*/; add(16, P); add(16, P) /*acc, acc_c*/; add(4, P) /*cnt*/;
    add(sizeof(ff_ray), P); add(4, P); add(sizeof(ff_hit), P); add(sizeof(ff_ray), 3ull * P); add(4, 3ull * P);
    add(4, (size_t)kKinds * P); add(4, 2 * kCtrStride); add(8, 8); add(4, 4); add(8, 4); add(8, 4);
    return b;
}

void ws_setup(FFWavefrontWS* ws, uint32_t P)
{
    if (ws->P == P && ws->buf.ptr) return;
    // a pool of another size: the allocation is kept when it is large enough
    // (freeing and allocating gigabytes costs milliseconds)
    ws->buf.alloc(ws_bytes(P));
    char* p = ws->buf.as<char>();
    WF& w = ws->w;
    w.P = P;
    w.samples_left = carve<uint32_t>(p, P);
    w.next_sample = carve<uint32_t>(p, P);
    w.key = carve<uint32_t>(p, P);
    w.length = carve<uint32_t>(p, P);
    w.phase = carve<uint32_t>(p, P);
    w.beta = carve<float4>(p, P);
    w.ray = carve<SlotRay>(p, P);
    w.shd = carve<SlotShade>(p, P);
    w.mis = carve<SlotMis>(p, P);
    w.vtx = carve<SlotVtx>(p, P);
    w.hit_ngeo = carve<float4>(p, P);
    w.acc = carve<float4>(p, P);
    w.acc_c = carve<float4>(p, P);
    w.cnt = carve<uint32_t>(p, P);
    w.ext_rays = carve<ff_ray>(p, P);
    w.ext_tag = carve<uint32_t>(p, P);
    w.ext_hits = carve<ff_hit>(p, P);
    ws->sh_rays_base[0] = w.sh_rays = carve<ff_ray>(p, 3ull * P);
    ws->sh_tag_base[0] = w.sh_tag = carve<uint32_t>(p, 3ull * P);
    w.mat_queue = carve<uint32_t>(p, (size_t)kKinds * P);
    ws->ctr_base = w.ctr = carve<uint32_t>(p, 2 * kCtrStride);
    w.defer = w.par = w.frame = 0u;
    w.totals = carve<unsigned long long>(p, 8);
    ws->err = carve<unsigned int>(p, 4);
    ws->trace_ctr = carve<unsigned long long>(p, 4);
    ws->fetch = carve<unsigned long long>(p, 4);
    ws->sh_rays_base[1] = nullptr;
    ws->sh_tag_base[1] = nullptr;
    w.pend = nullptr;
    w.vis2 = nullptr;
    ws->defer_P = 0;   // carved again by defer_setup, in its allocation if large enough
    ws->P = P;
}

// The deferred light terms' arrays (ff_render only, allocated on its first
// call for this pool size): the second frame parity's shadow queue, the
// pending records and the answer words of both parities.
void defer_setup(FFWavefrontWS* ws, uint32_t P)
{
    if (ws->defer_P == P && ws->defer_buf.ptr) return;
    size_t b = 0;
    auto add = [&](size_t sz, size_t n) { b += (sz * n + 255) & ~size_t(255); };
    add(sizeof(ff_ray), 3ull * P);
    add(4, 3ull * P);
    add(sizeof(SlotPend), 2ull * P);
    add(4, 2ull * P);
    ws->defer_buf.alloc(b);
    char* p = ws->defer_buf.as<char>();
    ws->sh_rays_base[1] = carve<ff_ray>(p, 3ull * P);
    ws->sh_tag_base[1] = carve<uint32_t>(p, 3ull * P);
    ws->w.pend = carve<SlotPend>(p, 2ull * P);
    ws->w.vis2 = carve<uint32_t>(p, 2ull * P);
    ws->defer_P = P;
}

}  // namespace

void ff_wavefront_render(ff_context* ctx, ff_scene* scene, const ff_render_settings* st, ff_film* film,
                         ff_render_stats* stats, const FFCacheHook* hook)
{
    FF_REQUIRE(st->spp > 0, "spp must be > 0");
    FF_REQUIRE(st->max_depth >= 1 && st->max_depth <= 64, "max_depth must be in [1, 64]");
    FF_REQUIRE(st->mode == FF_MODE_PARITY || st->mode == FF_MODE_CORRECTED, "unknown mode");
    ff_check_light(scene, st->light, st->mode);
    cudaStream_t stream = ctx->stream;
    const uint32_t WH = film->width * film->height;
    const uint64_t target = st->max_paths ? st->max_paths : kDefaultPoolTarget;
    uint32_t m = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(st->spp, target / WH));
    // shadow-ray tags are byte offsets into the SlotRay array (uint32): 32 * slot + 15 at most
    FF_REQUIRE((uint64_t)WH < (1ull << 27), "film too large for the path pool (at most 2^27 - 1 pixels)");
    while (m > 1 && (uint64_t)m * WH >= (1ull << 27)) --m;
    const uint32_t P = m * WH;
    if (!film->ws) film->ws = new FFWavefrontWS();
    FFWavefrontWS* ws = film->ws;
    ws_setup(ws, P);
    WF& w = ws->w;
    w.WH = WH;
    w.W = film->width;
    w.H = film->height;
    w.m = m;
    w.seed = st->seed;
    w.max_depth = st->max_depth;
    w.rr_depth = st->rr_depth;
    w.mode = st->mode;
    w.light = st->light;
    w.shadow_offset = st->shadow_offset > 0.f ? st->shadow_offset : 0.001f;
    w.shade = scene->shade.as<FFShadeTri>();
    w.tan = scene->tangent.as<FFTangentTri>();
    w.mats = scene->materials.as<ff_material>();
    w.area = scene->area_lights.as<ff_area_light>();
    w.n_area = scene->num_area_lights;
    w.tex = scene->tex_table.as<FFTexView>();
    w.env = ff_env_view(scene);
    w.lights = ff_light_set(scene, st->light, st->mode);
    w.cam = scene->camera;
    w.cache_mode = hook ? 1u : 0u;
    w.rough_threshold = hook ? hook->rough_threshold : 0.f;
    w.queries = hook ? static_cast<ffc::Record*>(hook->queries) : nullptr;
    w.n_queries = hook ? hook->n_queries : nullptr;
    if (hook) {
        FF_REQUIRE(hook->capacity >= P, "cache query buffer smaller than the path pool");
        FF_CUDA_CHECK(cudaMemsetAsync(hook->n_queries, 0, sizeof(uint32_t), stream));
    }
    const FFBvhView bvh = scene->view();

    // which material kinds occur
    std::vector<ff_material> mats(scene->num_materials);
    FF_CUDA_CHECK(cudaMemcpyAsync(mats.data(), scene->materials.ptr, sizeof(ff_material) * mats.size(),
                                  cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaMemsetAsync(w.totals, 0, 8 * sizeof(unsigned long long), stream));
    FF_CUDA_CHECK(cudaMemsetAsync(ws->err, 0, sizeof(unsigned int), stream));
    FF_CUDA_CHECK(cudaMemsetAsync(ws->fetch, 0, 4 * sizeof(unsigned long long), stream));
    FF_CUDA_CHECK(cudaStreamSynchronize(stream));
    bool kind_used[kKinds] = {false, false, false, false, false};
    for (auto& mt : mats) kind_used[mt.kind] = true;

    // deferred light terms: every render but the cached one (see the frame loop)
    const bool defer = hook == nullptr;
    if (defer) defer_setup(ws, P);
    w.defer = defer ? 1u : 0u;
    FF_CUDA_CHECK(cudaEventRecord(ctx->ev0, stream));
    k_init<<<(P + 255) / 256, 256, 0, stream>>>(w, st->spp, st->sample_offset);
    FF_CUDA_CHECK(cudaGetLastError());
    int shade_blocks = ctx->num_sms * 8;
    int n_kinds = 0;
    for (int k = 0; k < kKinds; ++k) n_kinds += kind_used[k] ? 1 : 0;
    // Optional per-stage timing: events around the stages of every frame.
    const bool profile = stats && (st->flags & FF_RENDER_PROFILE);
    std::vector<cudaEvent_t> evs;
    auto mark = [&](void) {
        if (!profile) return;
        cudaEvent_t e;
        FF_CUDA_CHECK(cudaEventCreate(&e));
        FF_CUDA_CHECK(cudaEventRecord(e, stream));
        evs.push_back(e);
    };
    uint32_t frames = 0;
    uint32_t active = 1;
    if (!ws->h_active) FF_CUDA_CHECK(cudaMallocHost(&ws->h_active, sizeof(uint32_t)));
    ws->ensure_streams();
    uint32_t* h_active = ws->h_active;
    const uint32_t max_frames = (st->spp + 1) * (st->max_depth + 2) + 8;
    // Deferred light terms (every render but the cached one): the any-hit
    // trace of frame f runs on the side stream beside k_logic, k_shade and
    // the closest-hit trace of frame f + 1, and k_logic of frame f + 2 adds
    // the light terms its answers let through.  Frames of one parity share
    // counters, a shadow queue and pending records, so frame f + 2 waits for
    // the any-hit trace of frame f.  Under stage timing everything stays on
    // the one stream.
    auto set_frame = [&](uint32_t f) -> uint32_t {
        const uint32_t par = defer ? (f & 1u) : 0u;
        w.par = par;
        w.frame = f;
        w.ctr = ws->ctr_base + kCtrStride * par;
        w.sh_rays = ws->sh_rays_base[par];
        w.sh_tag = ws->sh_tag_base[par];
        return par;
    };
    while (active && frames < max_frames) {
        // a batch of frames between host checks
        for (int b = 0; b < 4; ++b) {
            const uint32_t par = set_frame(frames);
            unsigned long long* tctr = ws->trace_ctr + 2 * par;
            uint8_t* occ = defer ? reinterpret_cast<uint8_t*>(w.vis2 + (size_t)par * P) : reinterpret_cast<uint8_t*>(w.ray);
            if (defer && !profile && frames >= 2) FF_CUDA_CHECK(cudaStreamWaitEvent(stream, ws->sh_done[par], 0));
            k_reset_counters<<<1, 32, 0, stream>>>(w.ctr, tctr);
            mark();
            k_logic<false><<<(P + 255) / 256, 256, 0, stream>>>(w);
            mark();
            // with stage timing (profile) every launch stays on the one stream
            FFWavefrontWS* side = profile ? nullptr : ws;
            const bool sel = w.lights.light == FF_LIGHT_ALL, corr = w.mode == FF_MODE_CORRECTED;
            // light selection needs the corrected mode (checked above)
            if (sel) launch_shade<true, false, true>(w, kind_used, shade_blocks, stream, side);
            else if (corr) launch_shade<false, false, true>(w, kind_used, shade_blocks, stream, side);
            else launch_shade<false, false, false>(w, kind_used, shade_blocks, stream, side);
            FF_CUDA_CHECK(cudaGetLastError());
            mark();
            if (profile) {
                // stage timing: the two traces one after the other
                ff_launch_trace_queue(ctx, bvh, w.ext_rays, w.ctr + C_EXT, P, w.ext_hits, false, tctr, ws->err,
                                      w.ext_tag, nullptr, nullptr, scene->refracts);
                mark();
                ff_launch_trace_queue(ctx, bvh, w.sh_rays, w.ctr + C_SH, 3ull * P, nullptr, true, tctr + 1, ws->err,
                                      w.sh_tag, occ);
                mark();
                // the traversal work of this frame's queues, counted by a second pass of the same
                // traversal (outside the stage marks)
                ff_launch_trace_count_queue(ctx, bvh, w.ext_rays, w.ctr + C_EXT, P, false, scene->refracts, ws->fetch,
                                            ws->err, stream);
                ff_launch_trace_count_queue(ctx, bvh, w.sh_rays, w.ctr + C_SH, 3ull * P, true, false, ws->fetch + 2,
                                            ws->err, stream);
            } else {
                // the traces are independent (hits by slot, answers by shadow-ray tag)
                FF_CUDA_CHECK(cudaEventRecord(ws->fork, stream));
                FF_CUDA_CHECK(cudaStreamWaitEvent(ws->side, ws->fork, 0));
                ff_launch_trace_queue(ctx, bvh, w.ext_rays, w.ctr + C_EXT, P, w.ext_hits, false, tctr, ws->err,
                                      w.ext_tag, nullptr, nullptr, scene->refracts);
                ff_launch_trace_queue(ctx, bvh, w.sh_rays, w.ctr + C_SH, 3ull * P, nullptr, true, tctr + 1, ws->err,
                                      w.sh_tag, occ, ws->side, false, defer ? kDeferShadowBlocks : 0);
                if (defer) {
                    FF_CUDA_CHECK(cudaEventRecord(ws->sh_done[par], ws->side));
                } else {
                    FF_CUDA_CHECK(cudaEventRecord(ws->join, ws->side));
                    FF_CUDA_CHECK(cudaStreamWaitEvent(stream, ws->join, 0));
                }
            }
            ++frames;
        }
        FF_CUDA_CHECK(cudaMemcpyAsync(h_active, w.ctr + C_ACTIVE, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        FF_CUDA_CHECK(cudaStreamSynchronize(stream));
        active = *h_active;
    }
    if (active) throw FFError{FF_ERR_INTERNAL, "wavefront did not finish within its frame bound"};
    if (defer) {
        // the light terms of the last two frames, once their any-hit traces are done
        if (!profile) {
            FF_CUDA_CHECK(cudaStreamWaitEvent(stream, ws->sh_done[0], 0));
            FF_CUDA_CHECK(cudaStreamWaitEvent(stream, ws->sh_done[1], 0));
        }
        for (uint32_t f = frames; f < frames + 2; ++f) {
            set_frame(f);
            k_flush_pending<<<(P + 255) / 256, 256, 0, stream>>>(w);
        }
        FF_CUDA_CHECK(cudaGetLastError());
    }
    // cache answers join their slots' sums before the film update
    if (hook) {
        if (hook->wait_before_query) FF_CUDA_CHECK(cudaStreamWaitEvent(stream, hook->wait_before_query, 0));
        if (hook->ev_query0) FF_CUDA_CHECK(cudaEventRecord(hook->ev_query0, stream));
        ff_cache_launch_infer(hook->cache, hook->queries, P, hook->n_queries, nullptr, w.acc);
        if (hook->ev_query1) FF_CUDA_CHECK(cudaEventRecord(hook->ev_query1, stream));
    }
    k_resolve<<<(WH + 255) / 256, 256, 0, stream>>>(w, film->accum.as<float4>(), film->comp.as<float4>(),
                                                   film->count.as<uint32_t>());
    FF_CUDA_CHECK(cudaGetLastError());
    FF_CUDA_CHECK(cudaEventRecord(ctx->ev1, stream));
    unsigned long long totals[3] = {0, 0, 0}, fetch[4] = {0, 0, 0, 0};
    unsigned int err = 0;
    FF_CUDA_CHECK(cudaMemcpyAsync(totals, w.totals, sizeof(totals), cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaMemcpyAsync(&err, ws->err, sizeof(err), cudaMemcpyDeviceToHost, stream));
    if (profile) FF_CUDA_CHECK(cudaMemcpyAsync(fetch, ws->fetch, sizeof(fetch), cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (err) throw FFError{FF_ERR_INTERNAL, "traversal exceeded its step bound (malformed BVH)"};
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->ext_nodes = fetch[0];
        stats->ext_tris = fetch[1];
        stats->shadow_nodes = fetch[2];
        stats->shadow_tris = fetch[3];
        if (profile) {
            // marks per frame: reset | logic | shade | trace ext | trace shadow
            const size_t per = 5;
            float t[4] = {0.f, 0.f, 0.f, 0.f};
            for (size_t f = 0; f + per <= evs.size(); f += per) {
                for (size_t k = 0; k + 1 < per; ++k) {
                    float x = 0.f;
                    cudaEventElapsedTime(&x, evs[f + k], evs[f + k + 1]);
                    t[k] += x;
                }
            }
            stats->ms_logic = t[0];
            stats->ms_shade = t[1];
            stats->ms_trace_extension = t[2];
            stats->ms_trace_shadow = t[3];
        }
        for (auto e : evs) cudaEventDestroy(e);
        // profiled renders add the two counting passes per frame
        // per frame: counter reset, logic, one shade per kind, two traces
        // (+ two counting passes when profiled); init and resolve; the flush
        stats->kernel_launches = frames * (4u + (uint32_t)n_kinds + (profile ? 2u : 0u)) + 2u + (defer ? 2u : 0u);
        stats->extension_rays = totals[0];
        stats->shadow_rays = totals[1];
        stats->samples = (uint64_t)st->spp * WH;
        stats->frames = frames;
        stats->ms_total = ms;
    }
}

namespace {

void adj_setup(FFWavefrontWS* ws, uint32_t P)
{
    WF& w = ws->w;
    if (ws->adj_P != P || !ws->adj_buf.ptr) {
        ws->adj_buf.release();
        size_t b = 0;
        auto add = [&](size_t sz) { b += (sz * P + 255) & ~size_t(255); };
        add(4);
        for (int k = 0; k < 6; ++k) add(16);
        add(8);
        ws->adj_buf.alloc(b);
        ws->adj_P = P;
    }
    char* p = ws->adj_buf.as<char>();
    w.pass = carve<uint32_t>(p, P);
    w.l_total = carve<float4>(p, P);
    w.v_albedo = carve<float4>(p, P);
    w.v_nee = carve<float4>(p, P);
    w.v_spec = carve<float4>(p, P);
    w.v_dext = carve<float4>(p, P);
    w.v_coef = carve<float4>(p, P);
}


}  // namespace

// The path-replay adjoint on the wavefront stages: every slot traces a
// sample as the primal pass, then replays it from its seed; gradients are
// scattered during the replay (k_logic<true>, k_shade<K, false, true>).
// The caller records the timing events, stages host buffers and reads the
// counters; this function leaves the stream unsynchronised except for the
// frame-loop checks.
void ff_wavefront_adjoint(ff_context* ctx, ff_scene* scene, const ff_render_settings* st, const FFAdjointTarget& t,
                          ff_render_stats* stats)
{
    FF_REQUIRE(st->max_depth >= 1 && st->max_depth <= 64, "max_depth must be in [1, 64]");
    FF_REQUIRE(st->light != FF_LIGHT_ALL, "the adjoint needs one light (FF_LIGHT_ALL is not supported)");
    cudaStream_t stream = ctx->stream;
    const uint32_t WH = t.width * t.height;
    const uint64_t target = st->max_paths ? st->max_paths : kDefaultPoolTarget;
    uint32_t m = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(st->spp, target / WH));
    // shadow-ray tags are byte offsets into the SlotRay array (uint32): 32 * slot + 15 at most
    FF_REQUIRE((uint64_t)WH < (1ull << 27), "film too large for the path pool (at most 2^27 - 1 pixels)");
    while (m > 1 && (uint64_t)m * WH >= (1ull << 27)) --m;
    const uint32_t P = m * WH;
    if (!ctx->adj_ws) ctx->adj_ws = new FFWavefrontWS();
    FFWavefrontWS* ws = ctx->adj_ws;
    ws_setup(ws, P);
    adj_setup(ws, P);
    WF& w = ws->w;
    w.WH = WH;
    w.W = t.width;
    w.H = t.height;
    w.m = m;
    w.seed = st->seed;
    w.max_depth = st->max_depth;
    w.rr_depth = st->rr_depth;
    w.mode = FF_MODE_CORRECTED;
    w.light = st->light;
    w.shadow_offset = st->shadow_offset > 0.f ? st->shadow_offset : 0.001f;
    w.shade = scene->shade.as<FFShadeTri>();
    w.tan = scene->tangent.as<FFTangentTri>();
    w.mats = scene->materials.as<ff_material>();
    w.area = scene->area_lights.as<ff_area_light>();
    w.n_area = scene->num_area_lights;
    w.tex = scene->tex_table.as<FFTexView>();
    w.env = ff_env_view(scene);
    w.lights = ff_light_set(scene, st->light, FF_MODE_CORRECTED);
    w.cam = scene->camera;
    w.cache_mode = 0u;
    w.rough_threshold = 0.f;
    w.queries = nullptr;
    w.n_queries = nullptr;
    // no deferred light terms: the replay needs each vertex's answers at the next frame
    w.defer = w.par = w.frame = 0u;
    w.ctr = ws->ctr_base;
    w.sh_rays = ws->sh_rays_base[0];
    w.sh_tag = ws->sh_tag_base[0];
    w.d_image = t.d_image;
    w.inv_spp = 1.f / (float)st->spp;
    w.adj_texture = t.texture;
    w.grad_tex = t.grad_tex;
    w.grad_env = t.grad_env;
    w.adj_rough = t.rough_texture;
    w.grad_rough = t.grad_rough;
    w.touched = t.touched;
    const FFBvhView bvh = scene->view();

    std::vector<ff_material> mats(scene->num_materials);
    FF_CUDA_CHECK(cudaMemcpyAsync(mats.data(), scene->materials.ptr, sizeof(ff_material) * mats.size(),
                                  cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaMemsetAsync(w.totals, 0, 8 * sizeof(unsigned long long), stream));
    FF_CUDA_CHECK(cudaMemsetAsync(ws->err, 0, sizeof(unsigned int), stream));
    FF_CUDA_CHECK(cudaStreamSynchronize(stream));
    bool kind_used[kKinds] = {false, false, false, false, false};
    for (auto& mt : mats) kind_used[mt.kind] = true;
    int n_kinds = 0;
    for (int k = 0; k < kKinds; ++k) n_kinds += kind_used[k] ? 1 : 0;

    k_init<<<(P + 255) / 256, 256, 0, stream>>>(w, st->spp, st->sample_offset);
    FF_CUDA_CHECK(cudaGetLastError());
    const int shade_blocks = ctx->num_sms * 8;
    // optional per-stage timing, as in ff_wavefront_render
    const bool profile = stats && (st->flags & FF_RENDER_PROFILE);
    std::vector<cudaEvent_t> evs;
    auto mark = [&](void) {
        if (!profile) return;
        cudaEvent_t e;
        FF_CUDA_CHECK(cudaEventCreate(&e));
        FF_CUDA_CHECK(cudaEventRecord(e, stream));
        evs.push_back(e);
    };
    uint32_t frames = 0;
    uint32_t active = 1;
    if (!ws->h_active) FF_CUDA_CHECK(cudaMallocHost(&ws->h_active, sizeof(uint32_t)));
    ws->ensure_streams();
    uint32_t* h_active = ws->h_active;
    // two passes per sample
    const uint32_t max_frames = 2 * (st->spp + 1) * (st->max_depth + 2) + 8;
    while (active && frames < max_frames) {
        for (int b = 0; b < 4; ++b) {
            k_reset_counters<<<1, 32, 0, stream>>>(w.ctr, ws->trace_ctr);
            mark();
            k_logic<true><<<(P + 255) / 256, 256, 0, stream>>>(w);
            mark();
            // side streams as in ff_wavefront_render (one stream under stage timing)
            launch_shade<false, true, true>(w, kind_used, shade_blocks, stream, profile ? nullptr : ws);
            FF_CUDA_CHECK(cudaGetLastError());
            mark();
            if (profile) {
                ff_launch_trace_queue(ctx, bvh, w.ext_rays, w.ctr + C_EXT, P, w.ext_hits, false, ws->trace_ctr,
                                      ws->err, w.ext_tag, nullptr, nullptr, scene->refracts);
                mark();
                ff_launch_trace_queue(ctx, bvh, w.sh_rays, w.ctr + C_SH, 3ull * P, nullptr, true,
                                      ws->trace_ctr + 1, ws->err, w.sh_tag, reinterpret_cast<uint8_t*>(w.ray));
                mark();
            } else {
                FF_CUDA_CHECK(cudaEventRecord(ws->fork, stream));
                FF_CUDA_CHECK(cudaStreamWaitEvent(ws->side, ws->fork, 0));
                ff_launch_trace_queue(ctx, bvh, w.ext_rays, w.ctr + C_EXT, P, w.ext_hits, false, ws->trace_ctr,
                                      ws->err, w.ext_tag, nullptr, nullptr, scene->refracts);
                ff_launch_trace_queue(ctx, bvh, w.sh_rays, w.ctr + C_SH, 3ull * P, nullptr, true,
                                      ws->trace_ctr + 1, ws->err, w.sh_tag, reinterpret_cast<uint8_t*>(w.ray),
                                      ws->side);
                FF_CUDA_CHECK(cudaEventRecord(ws->join, ws->side));
                FF_CUDA_CHECK(cudaStreamWaitEvent(stream, ws->join, 0));
            }
            ++frames;
        }
        FF_CUDA_CHECK(cudaMemcpyAsync(h_active, w.ctr + C_ACTIVE, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        FF_CUDA_CHECK(cudaStreamSynchronize(stream));
        active = *h_active;
    }
    if (active) throw FFError{FF_ERR_INTERNAL, "wavefront adjoint did not finish within its frame bound"};
    unsigned long long totals[2] = {0, 0};
    unsigned int err = 0;
    FF_CUDA_CHECK(cudaMemcpyAsync(totals, w.totals, sizeof(totals), cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaMemcpyAsync(&err, ws->err, sizeof(err), cudaMemcpyDeviceToHost, stream));
    FF_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (err) throw FFError{FF_ERR_INTERNAL, "traversal exceeded its step bound (malformed BVH)"};
    if (profile) {
        // 5 marks per frame: logic | shade | trace extension | trace shadow
        float t[4] = {0.f, 0.f, 0.f, 0.f};
        for (size_t f = 0; f + 5 <= evs.size(); f += 5) {
            for (int k = 0; k < 4; ++k) {
                float x = 0.f;
                cudaEventElapsedTime(&x, evs[f + k], evs[f + k + 1]);
                t[k] += x;
            }
        }
        stats->ms_logic = t[0];
        stats->ms_shade = t[1];
        stats->ms_trace_extension = t[2];
        stats->ms_trace_shadow = t[3];
    }
    for (auto e : evs) cudaEventDestroy(e);
    if (stats) {
        stats->kernel_launches = frames * (4u + (uint32_t)n_kinds) + 1u;   // counter reset, logic, shades, traces; init
        stats->extension_rays = totals[0];
        stats->shadow_rays = totals[1];
        stats->frames = frames;
    }
}
