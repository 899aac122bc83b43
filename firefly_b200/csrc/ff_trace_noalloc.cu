// ff_trace_noalloc.cu — ff_trace_host_noalloc: the host-pointer ray query
// with every byte of its device scratch in one file-scope __device__ array.
//
// Who needs it: callers that cannot allocate device memory.  An application
// whose device memory belongs to its own pool allocator under a fixed budget
// cannot have a library call cudaMalloc behind its back, and an interactive
// loop (picking under the cursor every frame, say) cannot take the implicit
// device-wide synchronisation of cudaMalloc / cudaFree.  ff_trace's host
// path grows its staging buffers with cudaMalloc; this entry point stages
// through a fixed array instead and never allocates.
//
// Scratch layout (kScratchBytes = 256 + FF_NOALLOC_MAX_RAYS * 48 bytes, about
// 3 MiB; every GPU that loads this library holds it until the process exits):
//   [0, 8)    work counter of the persistent trace kernel (zeroed every call)
//   [8, 12)   traversal error counter (zeroed every call)
//   [256, ..) FF_NOALLOC_MAX_RAYS rays (32 B each), then as many hits (16 B each)
//
// Every call on a device shares this one array and it keeps the last call's
// contents: the counters are cleared at the start of each call, the ray and
// hit areas are fully overwritten for the rays of the call.  Calls whose GPU
// work overlaps (two streams or two host threads on one device) race on the
// array; the caller must serialise them.
#include <mutex>

#include "ff_internal.h"

namespace {

constexpr size_t kHeaderBytes = 256;
constexpr size_t kScratchBytes = kHeaderBytes + (size_t)FF_NOALLOC_MAX_RAYS * (sizeof(ff_ray) + sizeof(ff_hit));

static __device__ __align__(256) unsigned char g_trace_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_trace_scratch on `dev`.  In host code the array's name
// is only a host-side stand-in; the device address comes from
// cudaGetSymbolAddress, taken once per device with that device current (the
// first call on each device does this, so it must not be the first call
// inside a stream capture).  The address stays cached for the life of the
// process: a cudaDeviceReset frees the array's device copy together with
// every context and scene of this library on that device, after which this
// entry point must not be called there.
unsigned char* scratch_on(int dev)
{
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (dev < 0 || dev >= kMaxDevices) throw FFError{FF_ERR_UNSUPPORTED, "device ordinal beyond the scratch table"};
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_trace_scratch);
        if (e != cudaSuccess || !p)
            throw FFError{FF_ERR_CUDA, std::string("cudaGetSymbolAddress(g_trace_scratch): ") + cudaGetErrorString(e)};
        g_scratch_addr[dev] = p;
    }
    return static_cast<unsigned char*>(g_scratch_addr[dev]);
}

}  // namespace

extern "C" ff_status ff_trace_host_noalloc(ff_context* ctx, const ff_scene* s, const ff_ray* rays, uint64_t n,
                                           ff_hit* hits, uint32_t flags)
{
    if (!ctx || !s) return FF_ERR_INVALID_ARG;
    if (s->ctx != ctx) {
        ctx->last_error = "scene belongs to another context";
        return FF_ERR_INVALID_ARG;
    }
    if (n > FF_NOALLOC_MAX_RAYS) {
        ctx->last_error = "ff_trace_host_noalloc: n = " + std::to_string(n) + " exceeds FF_NOALLOC_MAX_RAYS (" +
                          std::to_string(FF_NOALLOC_MAX_RAYS) + "); split the rays into calls of at most that many";
        return FF_ERR_INVALID_ARG;
    }
    if (flags & FF_MEM_DEVICE) {
        ctx->last_error = "ff_trace_host_noalloc takes host pointers; use ff_trace for device pointers";
        return FF_ERR_INVALID_ARG;
    }
    if (flags & FF_TRACE_TWO_SIDED) {
        ctx->last_error = "ff_trace_host_noalloc traces one-sided closest hits or any hits; use ff_trace for FF_TRACE_TWO_SIDED";
        return FF_ERR_INVALID_ARG;
    }
    if (n == 0) return FF_OK;
    if (!rays || !hits) return FF_ERR_INVALID_ARG;
    try {
        int prev = -1;
        FF_CUDA_CHECK(cudaGetDevice(&prev));
        if (prev != ctx->device) FF_CUDA_CHECK(cudaSetDevice(ctx->device));
        struct Restore {
            int dev, cur;
            ~Restore()
            {
                if (dev >= 0 && dev != cur) cudaSetDevice(dev);
            }
        } restore{prev, ctx->device};
        unsigned char* base = scratch_on(ctx->device);
        unsigned long long* counter = reinterpret_cast<unsigned long long*>(base);
        unsigned int* err = reinterpret_cast<unsigned int*>(base + 8);
        ff_ray* d_rays = reinterpret_cast<ff_ray*>(base + kHeaderBytes);
        ff_hit* d_hits = reinterpret_cast<ff_hit*>(base + kHeaderBytes + (size_t)FF_NOALLOC_MAX_RAYS * sizeof(ff_ray));
        cudaStream_t st = ctx->stream;
        FF_CUDA_CHECK(cudaMemsetAsync(base, 0, 16, st));
        FF_CUDA_CHECK(cudaMemcpyAsync(d_rays, rays, sizeof(ff_ray) * n, cudaMemcpyHostToDevice, st));
        ff_launch_trace_scratch(ctx, s, d_rays, n, d_hits, (flags & FF_TRACE_ANY) != 0, counter, err);
        FF_CUDA_CHECK(cudaMemcpyAsync(hits, d_hits, sizeof(ff_hit) * n, cudaMemcpyDeviceToHost, st));
        unsigned int h_err = 0;
        FF_CUDA_CHECK(cudaMemcpyAsync(&h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, st));
        FF_CUDA_CHECK(cudaStreamSynchronize(st));
        if (h_err) throw FFError{FF_ERR_INTERNAL, "traversal exceeded its step bound (malformed BVH)"};
        return FF_OK;
    } catch (const FFError& e) {
        ctx->last_error = e.msg;
        return e.status;
    } catch (...) {
        ctx->last_error = "unknown internal error";
        return FF_ERR_INTERNAL;
    }
}
