// ff_scene.cu — per-triangle shading attributes, materials, lights and
// textures uploaded at scene creation.
//
// Replaces the reference's mesh flattening into 200-byte dTriangle records
// (d_process_mesh + dTriangle::init, CUDA-RayTracer/kernel.cu:162-182,
// dTriangle.cu:22-32) and the managed-memory material / light tables
// (dScene.cpp:172-298).  Traversal reads only the 48-byte FFTri records;
// the attributes below are read once per hit, by original triangle index.
#include <cmath>
#include "ff_internal.h"
#include "ff_paths.cuh"
#include "ff_shade.cuh"

namespace {

__global__ void k_build_shading(const float3* __restrict__ pos, const uint3* __restrict__ idx,
                                const float3* __restrict__ nrm, const float2* __restrict__ uv,
                                const uint32_t* __restrict__ mat, uint32_t n, FFShadeTri* __restrict__ out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint3 t = idx[i];
    float3 v0 = pos[t.x], v1 = pos[t.y], v2 = pos[t.z];
    // dTriangle::init: face_normal = normalize(cross(v1 - v0, v2 - v0))
    float3 c = rn_cross(rn_sub(v1, v0), rn_sub(v2, v0));
    float l2 = rn_dot(c, c);
    float inv = 1.0f / sqrtf(l2);
    float3 fn = make_float3(c.x * inv, c.y * inv, c.z * inv);
    const float3 n0 = nrm ? nrm[t.x] : fn, n1 = nrm ? nrm[t.y] : fn, n2 = nrm ? nrm[t.z] : fn;
    const float2 zero = make_float2(0.f, 0.f);
    const float2 uv0 = uv ? uv[t.x] : zero, uv1 = uv ? uv[t.y] : zero, uv2 = uv ? uv[t.z] : zero;
    FFShadeTri s;
    s.n0x = n0.x, s.n0y = n0.y, s.n0z = n0.z;
    s.n1x = n1.x, s.n1y = n1.y, s.n1z = n1.z;
    s.n2x = n2.x, s.n2y = n2.y, s.n2z = n2.z;
    s.material = mat ? mat[i] : 0u;
    s.u0 = uv0.x, s.v0 = uv0.y, s.u1 = uv1.x, s.v1 = uv1.y, s.u2 = uv2.x, s.v2 = uv2.y;
    s.pad[0] = s.pad[1] = s.pad[2] = s.pad[3] = 0.f;
    out[i] = s;
}

// Tangent frames for normal textures.  With per-vertex tangents and
// bitangents (dVertex.cuh:8-9) each triangle takes its three vertices'.
// Without them the frame is derived per triangle from the texture
// coordinates: the edges e1 = v1 - v0 and e2 = v2 - v0 against their uv
// differences give T = (e1 dv2 - e2 dv1) / det and B = (e2 du1 - e1 du2) / det
// (det = du1 dv2 - du2 dv1; a degenerate uv mapping falls back to a frame
// around the face normal).  No reference counterpart for the derivation: the
// reference takes assimp's aiProcess_CalcTangentSpace frame.
__global__ void k_build_tangents(const float3* __restrict__ pos, const uint3* __restrict__ idx,
                                 const float2* __restrict__ uv, const float3* __restrict__ tan,
                                 const float3* __restrict__ bitan, uint32_t n, FFTangentTri* __restrict__ out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint3 t = idx[i];
    FFTangentTri f;
    if (tan && bitan) {
        f.t0 = tan[t.x];
        f.t1 = tan[t.y];
        f.t2 = tan[t.z];
        f.b0 = bitan[t.x];
        f.b1 = bitan[t.y];
        f.b2 = bitan[t.z];
    } else {
        const float3 v0 = pos[t.x], v1 = pos[t.y], v2 = pos[t.z];
        const float3 e1 = rn_sub(v1, v0), e2 = rn_sub(v2, v0);
        const float2 a = uv ? uv[t.x] : make_float2(0.f, 0.f), b = uv ? uv[t.y] : make_float2(0.f, 0.f),
                     c = uv ? uv[t.z] : make_float2(0.f, 0.f);
        const float du1 = b.x - a.x, dv1 = b.y - a.y, du2 = c.x - a.x, dv2 = c.y - a.y;
        const float det = du1 * dv2 - du2 * dv1;
        float3 T, B;
        if (fabsf(det) > 1e-20f) {
            const float r = 1.f / det;
            T = make_float3((e1.x * dv2 - e2.x * dv1) * r, (e1.y * dv2 - e2.y * dv1) * r, (e1.z * dv2 - e2.z * dv1) * r);
            B = make_float3((e2.x * du1 - e1.x * du2) * r, (e2.y * du1 - e1.y * du2) * r, (e2.z * du1 - e1.z * du2) * r);
        } else {
            const float3 nf = normalize3(rn_cross(e1, e2));
            T = normalize3(rn_cross(nf, fabsf(nf.x) > 0.5f ? make_float3(0.f, 1.f, 0.f) : make_float3(1.f, 0.f, 0.f)));
            B = rn_cross(nf, T);
        }
        f.t0 = f.t1 = f.t2 = T;
        f.b0 = f.b1 = f.b2 = B;
    }
    out[i] = f;
}

}  // namespace

void ff_build_env_tables(ff_context* ctx, ff_scene* s);

void ff_build_shading(ff_context* ctx, ff_scene* s, const ff_scene_desc* d, const float3* d_pos, const uint3* d_idx)
{
    cudaStream_t st = ctx->stream;
    const uint32_t n = d->num_triangles;
    DevBuf nrm, uv, mat;
    if (d->normals && d->num_vertices) {
        nrm.alloc(sizeof(float3) * d->num_vertices);
        FF_CUDA_CHECK(cudaMemcpyAsync(nrm.ptr, d->normals, sizeof(float3) * d->num_vertices, cudaMemcpyHostToDevice, st));
    }
    if (d->texcoords && d->num_vertices) {
        uv.alloc(sizeof(float2) * d->num_vertices);
        FF_CUDA_CHECK(cudaMemcpyAsync(uv.ptr, d->texcoords, sizeof(float2) * d->num_vertices, cudaMemcpyHostToDevice, st));
    }
    if (d->material_ids && n) {
        mat.alloc(sizeof(uint32_t) * n);
        FF_CUDA_CHECK(cudaMemcpyAsync(mat.ptr, d->material_ids, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
    }
    if (n) {
        s->shade.alloc(sizeof(FFShadeTri) * n);
        k_build_shading<<<(n + 255) / 256, 256, 0, st>>>(d_pos, d_idx, nrm.as<float3>(), uv.as<float2>(),
                                                         mat.as<uint32_t>(), n, s->shade.as<FFShadeTri>());
        FF_CUDA_CHECK(cudaGetLastError());
    }
    // Materials: a default grey FF_MAT_MIX when none are given.
    std::vector<ff_material> mats(d->materials, d->materials + d->num_materials);
    if (mats.empty()) {
        ff_material m{};
        m.base_color[0] = m.base_color[1] = m.base_color[2] = 0.5f;
        m.fresnel[0] = m.fresnel[1] = m.fresnel[2] = 0.04f;
        m.roughness = 1.f;
        m.ior = 1.5f;
        m.kind = FF_MAT_MIX;
        m.base_color_tex = m.roughness_tex = m.metallic_tex = m.metallic_roughness_tex = m.normal_tex = -1;
        mats.push_back(m);
    }
    // texture indices in range (the kernels index the texture table with them)
    for (const ff_material& mt : mats) {
        for (int32_t ti : {mt.base_color_tex, mt.roughness_tex, mt.metallic_tex, mt.metallic_roughness_tex,
                           mt.normal_tex})
            FF_REQUIRE(ti < (int32_t)d->num_textures, "material texture index out of range");
    }
    // tangent frames, only when some material has a normal texture
    bool normal_maps = false;
    for (const ff_material& mt : mats) normal_maps |= mt.normal_tex >= 0;
    FF_REQUIRE(!(d->tangents && !d->bitangents) && !(d->bitangents && !d->tangents),
               "tangents and bitangents come together");
    if (normal_maps && n) {
        DevBuf tg, btg;
        if (d->tangents && d->num_vertices) {
            tg.alloc(sizeof(float3) * d->num_vertices);
            btg.alloc(sizeof(float3) * d->num_vertices);
            FF_CUDA_CHECK(cudaMemcpyAsync(tg.ptr, d->tangents, sizeof(float3) * d->num_vertices,
                                          cudaMemcpyHostToDevice, st));
            FF_CUDA_CHECK(cudaMemcpyAsync(btg.ptr, d->bitangents, sizeof(float3) * d->num_vertices,
                                          cudaMemcpyHostToDevice, st));
        }
        s->tangent.alloc(sizeof(FFTangentTri) * n);
        k_build_tangents<<<(n + 255) / 256, 256, 0, st>>>(d_pos, d_idx, uv.as<float2>(), tg.as<float3>(),
                                                          btg.as<float3>(), n, s->tangent.as<FFTangentTri>());
        FF_CUDA_CHECK(cudaGetLastError());
        FF_CUDA_CHECK(cudaStreamSynchronize(st));   // tg / btg are freed on return
    } else {
        s->tangent.release();
    }
    s->num_materials = (uint32_t)mats.size();
    s->materials.alloc(sizeof(ff_material) * mats.size());
    FF_CUDA_CHECK(cudaMemcpyAsync(s->materials.ptr, mats.data(), sizeof(ff_material) * mats.size(),
                                  cudaMemcpyHostToDevice, st));
    // textures: one RGB float array each, plus a device table of views
    if (d->num_textures) {
        std::vector<FFTexView> views(d->num_textures);
        for (uint32_t i = 0; i < d->num_textures; ++i) {
            const ff_texture_desc& td = d->textures[i];
            FF_REQUIRE(td.rgb && td.width > 0 && td.height > 0, "texture without texels");
            DevBuf* b = new DevBuf();
            s->textures.push_back(b);
            b->alloc(sizeof(float3) * td.width * td.height);
            FF_CUDA_CHECK(cudaMemcpyAsync(b->ptr, td.rgb, sizeof(float3) * td.width * td.height, cudaMemcpyHostToDevice, st));
            views[i] = FFTexView{b->as<float3>(), (int)td.width, (int)td.height};
        }
        s->tex_table.alloc(sizeof(FFTexView) * views.size());
        FF_CUDA_CHECK(cudaMemcpyAsync(s->tex_table.ptr, views.data(), sizeof(FFTexView) * views.size(),
                                      cudaMemcpyHostToDevice, st));
        FF_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    s->num_area_lights = d->num_area_lights;
    if (d->num_area_lights) {
        s->area_lights.alloc(sizeof(ff_area_light) * d->num_area_lights);
        FF_CUDA_CHECK(cudaMemcpyAsync(s->area_lights.ptr, d->area_lights, sizeof(ff_area_light) * d->num_area_lights,
                                      cudaMemcpyHostToDevice, st));
    }
    // dDirectionalLight(dir) normalises its direction (dDirectionalLight.cu:10-14)
    s->num_dir_lights = d->num_directional_lights;
    if (d->num_directional_lights) {
        std::vector<ff_directional_light> dl(d->directional_lights, d->directional_lights + d->num_directional_lights);
        for (auto& l : dl) {
            const double x = l.direction[0], y = l.direction[1], z = l.direction[2];
            const double len = std::sqrt(x * x + y * y + z * z);
            FF_REQUIRE(len > 0.0 && std::isfinite(len), "directional light without a direction");
            l.direction[0] = (float)(x / len);
            l.direction[1] = (float)(y / len);
            l.direction[2] = (float)(z / len);
        }
        s->dir_lights.alloc(sizeof(ff_directional_light) * dl.size());
        FF_CUDA_CHECK(cudaMemcpyAsync(s->dir_lights.ptr, dl.data(), sizeof(ff_directional_light) * dl.size(),
                                      cudaMemcpyHostToDevice, st));
        FF_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    s->env.color = make_float3(d->env_color[0], d->env_color[1], d->env_color[2]);
    if (d->env_rgb) {
        s->env.width = (int)d->env_width;
        s->env.height = (int)d->env_height;
        s->env.rgb.alloc(sizeof(float3) * d->env_width * d->env_height);
        FF_CUDA_CHECK(cudaMemcpyAsync(s->env.rgb.ptr, d->env_rgb, sizeof(float3) * d->env_width * d->env_height,
                                      cudaMemcpyHostToDevice, st));
        ff_build_env_tables(ctx, s);
    }
    FF_CUDA_CHECK(cudaStreamSynchronize(st));
}

FFEnvView ff_env_view(const ff_scene* s)
{
    FFEnvView e;
    e.rgb = s->env.rgb.as<float3>();
    e.marginal = s->env.marginal.as<double>();
    e.cond = s->env.conditional.as<double>();
    e.guide_m = s->env.guide.as<uint32_t>();
    e.guide_c = e.guide_m ? e.guide_m + kGuideMarginal + 1 : nullptr;
    e.pdf = s->env.pdf.as<float>();
    e.width = s->env.width;
    e.height = s->env.height;
    e.color = s->env.color;
    e.radius = 10000.f;   // dEnvironmentLight.cu:14
    e.texel4 = s->env.texel4.as<float4>();
    return e;
}

void ff_check_light(const ff_scene* s, int32_t light, uint32_t mode)
{
    if (light == FF_LIGHT_ALL) {
        FF_REQUIRE(mode == FF_MODE_CORRECTED, "FF_LIGHT_ALL (light selection) needs FF_MODE_CORRECTED");
        FF_REQUIRE(s->env.width > 0 || s->num_area_lights + s->num_dir_lights > 0, "the scene has no light");
    } else if (light < 0) {
        FF_REQUIRE(light == -1, "light must be -1, FF_LIGHT_ALL or a light index");
        FF_REQUIRE(s->env.width > 0, "light -1 (environment) needs an environment map");
    } else {
        FF_REQUIRE((uint32_t)light < s->num_area_lights + s->num_dir_lights, "light index out of range");
    }
}

ffp::FFLightSet ff_light_set(const ff_scene* s, int32_t light, uint32_t mode)
{
    ffp::FFLightSet l;
    l.env = ff_env_view(s);
    l.has_env = s->env.width > 0;
    l.area = s->area_lights.as<ff_area_light>();
    l.n_area = s->num_area_lights;
    l.dirs = s->dir_lights.as<ff_directional_light>();
    l.n_dir = s->num_dir_lights;
    l.light = light;
    l.corrected = mode == FF_MODE_CORRECTED;
    return l;
}
