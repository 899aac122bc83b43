// ffrefcuda_harness.cu — the reference's own GPU ray traversal, unmodified,
// behind a C entry point.  TEST INFRASTRUCTURE ONLY (the "reference CUDA"
// baseline of the trace benchmark).
//
// The reference's dRay.cu and dTriangle.cu are compiled into this unit from
// the reference checkout (REF_DIR on the include path).  k_ref_extend and
// k_ref_shadow do what wf_extend / wf_shadow do (CUDA-RayTracer/kernel.cu:
// 488-543) for a plain array of rays: one thread per ray, 64 threads per
// block (kernel.cu:662), intersect() writing the 80-byte Isect per ray, and
// intersect_shadows() with the ray's tmax as its tmin bound (the visibility
// query of dDirectionalLight / dEnvironmentLight::visible).  The BVH and the
// reordered triangles come from the reference's own host build (BVHAccel,
// oracle/_ref/libffref.so).
#include "dRay.cu"
#include "dTriangle.cu"

namespace {

__global__ void k_ref_extend(const LinearBVHNode* nodes, const dTriangle* tris, const float* rays, long n, Isect* out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + 8 * i;
    dRay ray(make_float3(r[0], r[1], r[2]), make_float3(r[4], r[5], r[6]));
    Isect isect;
    intersect(nodes, tris, ray, isect);
    out[i] = isect;
}

__global__ void k_ref_shadow(const LinearBVHNode* nodes, const dTriangle* tris, const float* rays, long n,
                             unsigned char* occluded)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + 8 * i;
    dRay ray(make_float3(r[0], r[1], r[2]), make_float3(r[4], r[5], r[6]));
    float tmin = r[7];
    occluded[i] = intersect_shadows(nodes, tris, ray, tmin) ? 1 : 0;
}

}  // namespace

extern "C" {

int ffrefcuda_sizes(int* node_bytes, int* tri_bytes, int* isect_bytes)
{
    *node_bytes = (int)sizeof(LinearBVHNode);
    *tri_bytes = (int)sizeof(dTriangle);
    *isect_bytes = (int)sizeof(Isect);
    return 0;
}

// rays: n x 8 floats (o, tmin, d, tmax) in host memory.  Closest-hit (any = 0):
// t_out = Isect.distance (inf when not found), prim_out = the reference's
// post-reorder triangle index or -1.  Any-hit: prim_out = 1 when occluded,
// else -1.  The launch is repeated `reps` times; ms_out = mean device time of
// one launch (CUDA events).  Returns 0, or a cudaError_t.
int ffrefcuda_trace(const void* nodes, int num_nodes, const void* tris, int num_tris, const float* rays, long n,
                    float* t_out, int* prim_out, int any, int reps, float* ms_out)
{
    LinearBVHNode* d_nodes = nullptr;
    dTriangle* d_tris = nullptr;
    float* d_rays = nullptr;
    Isect* d_isect = nullptr;
    unsigned char* d_occ = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaSuccess;
    std::vector<Isect> isect;
    std::vector<unsigned char> occ;
#define FFR_TRY(x)                \
    do {                          \
        err = (x);                \
        if (err != cudaSuccess) { \
            goto done;            \
        }                         \
    } while (0)
    FFR_TRY(cudaMalloc(&d_nodes, sizeof(LinearBVHNode) * (size_t)num_nodes));
    FFR_TRY(cudaMalloc(&d_tris, sizeof(dTriangle) * (size_t)num_tris));
    FFR_TRY(cudaMalloc(&d_rays, sizeof(float) * 8 * (size_t)n));
    FFR_TRY(cudaMemcpy(d_nodes, nodes, sizeof(LinearBVHNode) * (size_t)num_nodes, cudaMemcpyHostToDevice));
    FFR_TRY(cudaMemcpy(d_tris, tris, sizeof(dTriangle) * (size_t)num_tris, cudaMemcpyHostToDevice));
    FFR_TRY(cudaMemcpy(d_rays, rays, sizeof(float) * 8 * (size_t)n, cudaMemcpyHostToDevice));
    if (any) FFR_TRY(cudaMalloc(&d_occ, (size_t)n));
    else FFR_TRY(cudaMalloc(&d_isect, sizeof(Isect) * (size_t)n));
    FFR_TRY(cudaEventCreate(&e0));
    FFR_TRY(cudaEventCreate(&e1));
    {
        const int block = 64;
        const unsigned grid = (unsigned)((n + block - 1) / block);
        // one untimed launch, then `reps` timed ones
        for (int k = -1; k < reps; ++k) {
            if (k == 0) FFR_TRY(cudaEventRecord(e0));
            if (any) k_ref_shadow<<<grid, block>>>(d_nodes, d_tris, d_rays, n, d_occ);
            else k_ref_extend<<<grid, block>>>(d_nodes, d_tris, d_rays, n, d_isect);
            FFR_TRY(cudaGetLastError());
        }
        FFR_TRY(cudaEventRecord(e1));
        FFR_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms_out) *ms_out = reps > 0 ? ms / (float)reps : 0.f;
    }
    if (any) {
        occ.resize((size_t)n);
        FFR_TRY(cudaMemcpy(occ.data(), d_occ, (size_t)n, cudaMemcpyDeviceToHost));
        for (long i = 0; i < n; ++i) prim_out[i] = occ[(size_t)i] ? 1 : -1;
    } else {
        isect.resize((size_t)n);
        FFR_TRY(cudaMemcpy(isect.data(), d_isect, sizeof(Isect) * (size_t)n, cudaMemcpyDeviceToHost));
        for (long i = 0; i < n; ++i) {
            t_out[i] = isect[(size_t)i].wasFound ? isect[(size_t)i].distance : INFINITY;
            prim_out[i] = isect[(size_t)i].wasFound ? isect[(size_t)i].triangle_id : -1;
        }
    }
done:
#undef FFR_TRY
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_nodes);
    cudaFree(d_tris);
    cudaFree(d_rays);
    cudaFree(d_isect);
    cudaFree(d_occ);
    return (int)err;
}

}  // extern "C"
