// ff_trace.cu — persistent closest-hit / any-hit trace kernel behind ff_trace.
//
// Replaces wf_extend / wf_shadow (CUDA-RayTracer/kernel.cu:488-543), which
// launch one thread per queued ray over a binary BVH with a 64-entry local
// stack.  Here every warp is persistent: idle lanes take new rays from a
// global counter with one warp-aggregated atomic, so lanes whose rays finish
// early are refilled instead of idling until the slowest ray of the warp ends
// (Aila & Laine 2009, "Understanding the efficiency of ray traversal on GPUs").
#include "ff_internal.h"
#include "ff_trace.cuh"

static_assert(kMaxStack == kMaxStackDepth, "stack size must match the build-time depth check");

namespace {

constexpr int kTraceBlock = 128;
// Refill when at least this many lanes of the warp are idle.
constexpr int kRefillIdle = 8;

// Output: hits[ray] for every ray, or, with tags (the wavefront's queues),
// per the ray's tag: a closest hit goes to hits[tag] (tag = the path slot, so
// the next stage reads its hit in slot order without the queue index), an
// any-hit answer to occ[tag] (1 occluded, 0 clear; tag = 4 * slot + shadow
// ray index, so the next stage reads one 4-byte word of answers per slot).
//
// TWO (closest hit only): rays whose tmin carries the sign bit are traced
// two-sided (ff_test_tri_closest); a back-face hit reports prim = -2 - index.
template <bool ANY, bool TAGGED, bool TWO = false>
__global__ void __launch_bounds__(kTraceBlock, 8)
    k_trace(FFBvhView bvh, const ff_ray* __restrict__ rays, ff_hit* __restrict__ hits, uint64_t n,
            unsigned long long* __restrict__ counter, unsigned int* __restrict__ err,
            const uint32_t* __restrict__ n_dev, const uint32_t* __restrict__ tags, uint8_t* __restrict__ occ)
{
    // Queue-driven launches (the wavefront) read the ray count written by the
    // producing stage; n is then the queue capacity.
    if (n_dev) n = min(n, (uint64_t)*n_dev);
    // A ray visits every node at most once; more steps than nodes means a
    // malformed BVH.  The ray is then ended and counted in err[0] instead of
    // looping.
    const uint32_t max_steps = bvh.num_nodes + 2u;
    __shared__ uint2 s_stack[kShortStack * kTraceBlock];
    FFStack st;
    st.sm = s_stack + threadIdx.x;
    st.stride = kTraceBlock;
    st.sp = 0;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;

    FFRayState r;
    uint2 cur = make_uint2(0u, 0u);
    uint64_t ray_id = 0;
    uint32_t tag = 0;
    uint32_t steps = 0;
    bool active = false;
    bool exhausted = false;

    while (true) {
        // Refill idle lanes with new rays.
        const uint32_t want = __ballot_sync(0xffffffffu, !active && !exhausted);
        if (want) {
            const uint32_t leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(want));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!active && !exhausted) {
                ray_id = base + __popc(want & lt_mask);
                if (ray_id < n) {
                    const float4 r0 = __ldg(reinterpret_cast<const float4*>(rays + ray_id));
                    const float4 r1 = __ldg(reinterpret_cast<const float4*>(rays + ray_id) + 1);
                    if (TAGGED) tag = __ldg(tags + ray_id);
                    // untagged two-sided launches (ff_trace with FF_TRACE_TWO_SIDED) mark every ray;
                    // tagged ones (the wavefront) carry the mark in each ray's tmin
                    const float tmin = (TWO && !TAGGED) ? -(r0.w > 0.f ? r0.w : 0.f) : r0.w;
                    ff_ray_setup(r, make_float3(r0.x, r0.y, r0.z), make_float3(r1.x, r1.y, r1.z), tmin, r1.w, ANY);
                    cur = ff_root_group(r);
                    st.reset();
                    steps = 0;
                    active = bvh.num_nodes > 0;
                    if (!active) {
                        if (!TAGGED) hits[ray_id] = ff_hit{r.tmax, 0.f, 0.f, -1};
                        else if (ANY) occ[tag] = 0;
                        else hits[tag] = ff_hit{r.tmax, 0.f, 0.f, -1};
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) {
            if (__all_sync(0xffffffffu, exhausted)) break;
            continue;
        }
        // Traverse until enough lanes are idle to make a refill worthwhile.
        while (true) {
            if (active) {
                const bool done = ff_traverse_step<ANY, TWO>(bvh, r, cur, st);
                if (st.overflow || ++steps > max_steps) atomicAdd(err, 1u);
                if (done || steps > max_steps) {
                    const int32_t prim = TWO ? ff_hit_of(r).prim : (r.prim == 0xffffffffu ? -1 : (int32_t)r.prim);
                    const float4 out = make_float4(r.tmax, r.u, r.v, __int_as_float(prim));
                    if (!TAGGED) *reinterpret_cast<float4*>(hits + ray_id) = out;
                    else if (ANY) occ[tag] = prim >= 0 ? 1 : 0;
                    else *reinterpret_cast<float4*>(hits + tag) = out;
                    active = false;
                }
            }
            const uint32_t idle = __ballot_sync(0xffffffffu, !active && !exhausted);
            const uint32_t busy = __ballot_sync(0xffffffffu, active);
            if (busy == 0u || __popc(idle) >= kRefillIdle) break;
        }
    }
}

// Traversal work of n rays (ff_trace_count): one thread per ray over the same
// traversal step as k_trace, so each ray visits the same nodes and tests the
// same triangles; out[0] += node records fetched, out[1] += triangles tested.
// QUEUE: a wavefront queue whose length is in n_dev (n its capacity), whose
// rays carry their own two-sided mark (as k_trace<*, tagged> reads them).
template <bool ANY, bool TWO = false, bool QUEUE = false>
__global__ void __launch_bounds__(kTraceBlock) k_trace_count(FFBvhView bvh, const ff_ray* __restrict__ rays,
                                                             uint64_t n, unsigned long long* __restrict__ out,
                                                             unsigned int* __restrict__ err,
                                                             const uint32_t* __restrict__ n_dev = nullptr)
{
    if (QUEUE) n = min(n, (uint64_t)*n_dev);
    __shared__ uint2 s_stack[kShortStack * kTraceBlock];
    FFStack st;
    st.sm = s_stack + threadIdx.x;
    st.stride = kTraceBlock;
    st.sp = 0;
    FFCount count;
    const uint32_t max_steps = bvh.num_nodes + 2u;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!bvh.num_nodes) break;
        const float4 r0 = __ldg(reinterpret_cast<const float4*>(rays + i));
        const float4 r1 = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
        FFRayState r;
        const float tmin = (TWO && !QUEUE) ? -(r0.w > 0.f ? r0.w : 0.f) : r0.w;
        ff_ray_setup(r, make_float3(r0.x, r0.y, r0.z), make_float3(r1.x, r1.y, r1.z), tmin, r1.w, ANY);
        uint2 cur = ff_root_group(r);
        st.reset();
        uint32_t steps = 0;
        while (!ff_traverse_step<ANY, FFCount, TWO>(bvh, r, cur, st, count)) {
            if (st.overflow || ++steps > max_steps) {
                atomicAdd(err, 1u);
                break;
            }
        }
    }
    unsigned long long a = count.nodes, b = count.tris;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(out, a);
        atomicAdd(out + 1, b);
    }
}

}  // namespace

void ff_launch_trace_count(ff_context* ctx, const ff_scene* s, const ff_ray* d_rays, uint64_t n, bool any_hit,
                           unsigned long long* d_out, unsigned int* err, bool two_sided)
{
    if (n == 0) return;
    uint64_t grid = (uint64_t)ctx->num_sms * 8;
    const uint64_t need = (n + kTraceBlock - 1) / kTraceBlock;
    if (grid > need) grid = need;
    if (any_hit)
        k_trace_count<true><<<(unsigned)grid, kTraceBlock, 0, ctx->stream>>>(s->view(), d_rays, n, d_out, err);
    else if (two_sided)
        k_trace_count<false, true><<<(unsigned)grid, kTraceBlock, 0, ctx->stream>>>(s->view(), d_rays, n, d_out, err);
    else
        k_trace_count<false><<<(unsigned)grid, kTraceBlock, 0, ctx->stream>>>(s->view(), d_rays, n, d_out, err);
    FF_CUDA_CHECK(cudaGetLastError());
}

void ff_launch_trace_count_queue(ff_context* ctx, const FFBvhView& bvh, const ff_ray* d_rays, const uint32_t* n_dev,
                                 uint64_t cap, bool any_hit, bool two_sided, unsigned long long* d_out,
                                 unsigned int* err, cudaStream_t stream)
{
    if (cap == 0) return;
    uint64_t grid = (uint64_t)ctx->num_sms * 8;
    const uint64_t need = (cap + kTraceBlock - 1) / kTraceBlock;
    if (grid > need) grid = need;
    const dim3 g((unsigned)grid), b(kTraceBlock);
    if (any_hit)
        k_trace_count<true, false, true><<<g, b, 0, stream>>>(bvh, d_rays, cap, d_out, err, n_dev);
    else if (two_sided)
        k_trace_count<false, true, true><<<g, b, 0, stream>>>(bvh, d_rays, cap, d_out, err, n_dev);
    else
        k_trace_count<false, false, true><<<g, b, 0, stream>>>(bvh, d_rays, cap, d_out, err, n_dev);
    FF_CUDA_CHECK(cudaGetLastError());
}

void ff_launch_trace(ff_context* ctx, const ff_scene* s, const ff_ray* d_rays, uint64_t n, ff_hit* d_hits,
                     bool any_hit, bool two_sided)
{
    if (n == 0) return;
    unsigned long long* counter = ctx->counters.as<unsigned long long>();
    // counters: [0..7] ray counter, [8..11] traversal error count (sticky
    // until read by ff_trace_errors / the host-pointer path)
    unsigned int* err = reinterpret_cast<unsigned int*>(ctx->counters.as<char>() + 8);
    FF_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), ctx->stream));
    const void* fn = any_hit ? (const void*)k_trace<true, false>
                             : (two_sided ? (const void*)k_trace<false, false, true> : (const void*)k_trace<false, false>);
    int blocks_per_sm = 0;
    FF_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, fn, kTraceBlock, 0));
    blocks_per_sm = blocks_per_sm < 1 ? 1 : blocks_per_sm;
    uint64_t grid = (uint64_t)ctx->num_sms * blocks_per_sm;
    const uint64_t need = (n + kTraceBlock - 1) / kTraceBlock;
    if (grid > need) grid = need;
    if (any_hit)
        k_trace<true, false><<<(unsigned)grid, kTraceBlock, 0, ctx->stream>>>(s->view(), d_rays, d_hits, n, counter,
                                                                              err, nullptr, nullptr, nullptr);
    else if (two_sided)
        k_trace<false, false, true><<<(unsigned)grid, kTraceBlock, 0, ctx->stream>>>(
            s->view(), d_rays, d_hits, n, counter, err, nullptr, nullptr, nullptr);
    else
        k_trace<false, false><<<(unsigned)grid, kTraceBlock, 0, ctx->stream>>>(s->view(), d_rays, d_hits, n, counter,
                                                                              err, nullptr, nullptr, nullptr);
    FF_CUDA_CHECK(cudaGetLastError());
}

// Same launch as ff_launch_trace, with the work counter and the error counter
// supplied by the caller instead of taken from the context's allocation.
void ff_launch_trace_scratch(ff_context* ctx, const ff_scene* s, const ff_ray* d_rays, uint64_t n, ff_hit* d_hits,
                             bool any_hit, unsigned long long* counter, unsigned int* err)
{
    if (n == 0) return;
    int blocks_per_sm = 0;
    if (any_hit)
        FF_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_trace<true, false>, kTraceBlock, 0));
    else
        FF_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_trace<false, false>, kTraceBlock, 0));
    blocks_per_sm = blocks_per_sm < 1 ? 1 : blocks_per_sm;
    uint64_t grid = (uint64_t)ctx->num_sms * blocks_per_sm;
    const uint64_t need = (n + kTraceBlock - 1) / kTraceBlock;
    if (grid > need) grid = need;
    if (any_hit)
        k_trace<true, false><<<(unsigned)grid, kTraceBlock, 0, ctx->stream>>>(s->view(), d_rays, d_hits, n, counter,
                                                                              err, nullptr, nullptr, nullptr);
    else
        k_trace<false, false><<<(unsigned)grid, kTraceBlock, 0, ctx->stream>>>(s->view(), d_rays, d_hits, n, counter,
                                                                              err, nullptr, nullptr, nullptr);
    FF_CUDA_CHECK(cudaGetLastError());
}

// Trace a device-resident queue whose length the previous stage wrote to
// n_dev (at most cap rays), on the context's stream.  counter must be zeroed
// by the caller before the launch.  two_sided (closest hit only): the
// kernel honours the per-ray two-sided mark (the sign bit of tmin).
void ff_launch_trace_queue(ff_context* ctx, const FFBvhView& bvh, const ff_ray* d_rays, const uint32_t* n_dev,
                           uint64_t cap, ff_hit* d_hits, bool any_hit, unsigned long long* counter, unsigned int* err,
                           const uint32_t* tags, uint8_t* occ, cudaStream_t stream, bool two_sided, int max_blocks_per_sm)
{
    if (cap == 0) return;
    const bool two = two_sided && !any_hit;
    using Kernel = void (*)(FFBvhView, const ff_ray*, ff_hit*, uint64_t, unsigned long long*, unsigned int*,
                            const uint32_t*, const uint32_t*, uint8_t*);
    const Kernel fn = any_hit ? (tags ? k_trace<true, true> : k_trace<true, false>)
                              : (tags ? (two ? k_trace<false, true, true> : k_trace<false, true>)
                                      : (two ? k_trace<false, false, true> : k_trace<false, false>));
    // occupancy of the variant launched, on the context's device; calls on
    // one context are externally synchronised, so the per-context cache
    // needs no lock
    int& blocks_per_sm = ctx->trace_bps[(any_hit ? 1 : 0) | (tags ? 2 : 0) | (two ? 4 : 0)];
    if (blocks_per_sm == 0) {
        int b = 0;
        FF_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kTraceBlock, 0));
        blocks_per_sm = b < 1 ? 1 : b;
    }
    const int bps = max_blocks_per_sm > 0 && max_blocks_per_sm < blocks_per_sm ? max_blocks_per_sm : blocks_per_sm;
    uint64_t grid = (uint64_t)ctx->num_sms * bps;
    const uint64_t need = (cap + kTraceBlock - 1) / kTraceBlock;
    if (grid > need) grid = need;
    cudaStream_t st = stream ? stream : ctx->stream;
    fn<<<dim3((unsigned)grid), dim3(kTraceBlock), 0, st>>>(bvh, d_rays, d_hits, cap, counter, err, n_dev, tags, occ);
    FF_CUDA_CHECK(cudaGetLastError());
}
