// UV-space maps of the renderer (compute_normal_map = normal / position / face).
//
// Reference: CudaRenderer/cpp/src/Renderer/CUDABasedRasterization.cpp:187-330
// (texel table, built on the host with OpenMP on the first forward call) and
// CUDABasedRasterization.cu:458-549 (renderNormalMapDevice).  In these modes
// the reference op does not rasterise the views at all: the face, barycentric
// and render buffers keep their initial values (-1, 0, 0) and only the vertex
// normals and the UV map are written (CUDABasedRasterization.cu:562-575).
//
// The texel table maps every texel centre to the triangle whose UV triangle
// contains it and the barycentrics of the texel in that triangle.  Here it is
// built on the device, once per texture size: one thread per triangle visits
// the texels of its UV bounding box (widened by 2 texels, as in the
// reference) with the reference's host ray test, keeping the largest face id
// per texel (the last writer of the reference's loop in serial order; its
// OpenMP loop leaves texels on shared UV edges to whichever thread writes
// last), then one thread per texel recomputes the barycentrics of the winner.
// The host ray test runs without fused multiply-adds (x86-64 SSE code), so
// its arithmetic is written here with explicitly rounded single operations.
#include "renderer.cuh"

namespace hc {
namespace {

// host float arithmetic: every product and sum rounded on its own
struct HF3 {
    float x, y, z;
};
__device__ __forceinline__ HF3 hf3(float x, float y, float z) { return HF3{x, y, z}; }
__device__ __forceinline__ HF3 hsub(HF3 a, HF3 b) { return hf3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ HF3 hadd(HF3 a, HF3 b) { return hf3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ HF3 hscale(float s, HF3 a) { return hf3(__fmul_rn(s, a.x), __fmul_rn(s, a.y), __fmul_rn(s, a.z)); }
__device__ __forceinline__ HF3 hdiv(HF3 a, float s) { return hf3(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)); }
__device__ __forceinline__ float hdot(HF3 a, HF3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ HF3 hcross(HF3 a, HF3 b) {
    return hf3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
               __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// rayTriangleIntersectHost (CUDABasedRasterization.cpp:187-262) for the
// texel ray: origin (x + 0.5, y + 0.5, 1), direction (0, 0, -1), triangle in
// texel units with z = 0.
__device__ bool texel_hit(HF3 o, HF3 v0, HF3 v1, HF3 v2, float& a, float& b) {
    v0 = hdiv(v0, 1000.f);
    v1 = hdiv(v1, 1000.f);
    v2 = hdiv(v2, 1000.f);
    o = hdiv(o, 1000.f);
    const HF3 dir = hf3(0.f, 0.f, -1.f);
    const HF3 N = hcross(hsub(v1, v0), hsub(v2, v0));
    const float ndr = hdot(dir, N);
    if (fabsf(ndr) < 0.0000001f) return false;
    const float t = __fdiv_rn(__fsub_rn(hdot(v0, N), hdot(o, N)), ndr);
    if (t < 0.f) return false;
    const HF3 P = hadd(o, hscale(t, dir));
    if (hdot(N, hcross(hsub(v1, v0), hsub(P, v0))) < 0.f) return false;
    if ((a = hdot(N, hcross(hsub(v2, v1), hsub(P, v1)))) < 0.f) return false;
    if ((b = hdot(N, hcross(hsub(v0, v2), hsub(P, v2)))) < 0.f) return false;
    const float denom = hdot(N, N);
    a = __fdiv_rn(a, denom);
    b = __fdiv_rn(b, denom);
    return true;
}

__device__ __forceinline__ void uv_corners(const float* tc, int f, int tw, int th, HF3& t0, HF3& t1, HF3& t2) {
    const float* c = tc + 6LL * f;
    t0 = hf3(__fmul_rn((float)tw, c[0]), __fmul_rn((float)th, __fsub_rn(1.f, c[1])), 0.f);
    t1 = hf3(__fmul_rn((float)tw, c[2]), __fmul_rn((float)th, __fsub_rn(1.f, c[3])), 0.f);
    t2 = hf3(__fmul_rn((float)tw, c[4]), __fmul_rn((float)th, __fsub_rn(1.f, c[5])), 0.f);
}

__global__ void k_texel_faces(int F, int tw, int th, const float* __restrict__ tc, int* __restrict__ texel_face) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    HF3 t0, t1, t2;
    uv_corners(tc, f, tw, th, t0, t1, t2);
    const int x0 = (int)fmaxf(fminf(t0.x, fminf(t1.x, t2.x)) - 2.f, 0.f);
    const int x1 = (int)fminf(fmaxf(t0.x, fmaxf(t1.x, t2.x)) + 2.f, (float)tw);
    const int y0 = (int)fmaxf(fminf(t0.y, fminf(t1.y, t2.y)) - 2.f, 0.f);
    const int y1 = (int)fminf(fmaxf(t0.y, fmaxf(t1.y, t2.y)) + 2.f, (float)th);
    for (int x = x0; x < x1; ++x)
        for (int y = y0; y < y1; ++y) {
            float a, b;
            if (texel_hit(hf3(x + 0.5f, y + 0.5f, 1.f), t0, t1, t2, a, b)) atomicMax(texel_face + y * tw + x, f);
        }
}

// (face, a, b, c) per texel; (0, 0, 0, 0) where no triangle covers it
__global__ void k_texel_table(int tw, int th, const float* __restrict__ tc, const int* __restrict__ texel_face,
                              float4* __restrict__ table) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tw * th) return;
    const int f = texel_face[i];
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (f >= 0) {
        HF3 t0, t1, t2;
        uv_corners(tc, f, tw, th, t0, t1, t2);
        float a = 0.f, b = 0.f;
        texel_hit(hf3(i % tw + 0.5f, i / tw + 0.5f, 1.f), t0, t1, t2, a, b);
        r = make_float4((float)f, a, b, __fsub_rn(__fsub_rn(1.f, a), b));
    }
    table[i] = r;
}

// renderNormalMapDevice (CUDABasedRasterization.cu:458-549) per (frame, texel):
// normal = barycentric blend of the normalised vertex normals of camera 0,
// normalised; position = blend of the vertex positions; face = the face id.
__global__ void k_uv_map(int B, int C, int N, int n_texels, int mode, const int3* __restrict__ faces,
                         const float4* __restrict__ table, const float* __restrict__ verts,
                         const float* __restrict__ vnormal, float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * n_texels) return;
    const int b = (int)(i / n_texels), p = (int)(i % n_texels);
    const float4 info = table[p];
    float3 r;
    if (mode == kNmFace) {
        r = make_float3(info.x, info.x, info.x);
    } else {
        const int3 id = faces[(int)info.x];
        const float* src = mode == kNmOriginal ? vnormal + (long long)b * C * N * 3 : verts + (long long)b * N * 3;
        float3 v0 = ld3(src + 3 * id.x), v1 = ld3(src + 3 * id.y), v2 = ld3(src + 3 * id.z);
        if (mode == kNmOriginal) {
            if (length3(v0) != 0.f) v0 = v0 / length3(v0);
            if (length3(v1) != 0.f) v1 = v1 / length3(v1);
            if (length3(v2) != 0.f) v2 = v2 / length3(v2);
        }
        r = v0 * info.y + v1 * info.z + v2 * info.w;
        if (mode == kNmOriginal && length3(r) != 0.f) r = r / length3(r);
    }
    st3(out + 3 * i, r);
}

}  // namespace

__global__ void k_vertex_normals(int B, int C, int N, const int3* __restrict__ faces, const int* __restrict__ vf,
                                 const int2* __restrict__ vf_id, const float* __restrict__ verts,
                                 float* __restrict__ out);

hc_status raster_uv_maps(const Topology& topo, UvTable& tab, cudaStream_t s, int B, int C, long long P_frame, int mode,
                         const float* verts, int tex_h, int tex_w, float* bary, int* face, float* render,
                         float* vnormal, float* uv_map) {
    HC_REQUIRE(topo.has_texcoords, "compute_normal_map needs texture_coordinates");
    HC_REQUIRE(tex_h > 0 && tex_w > 0, "compute_normal_map needs the texture size");
    HC_REQUIRE(uv_map, "compute_normal_map needs the normal_map output");
    const long long px = (long long)B * P_frame;
    HC_CUDA(cudaMemsetAsync(face, 0xff, sizeof(int) * px, s));
    HC_CUDA(cudaMemsetAsync(bary, 0, sizeof(float) * 2 * px, s));
    HC_CUDA(cudaMemsetAsync(render, 0, sizeof(float) * 3 * px, s));
    const int N = topo.N, F = topo.F;
    k_vertex_normals<<<div_up((long long)B * N, 256), 256, 0, s>>>(B, C, N, topo.faces.as<int3>(), topo.vf.as<int>(),
                                                                    topo.vf_id.as<int2>(), verts, vnormal);
    HC_CHECK_LAUNCH();
    const int nt = tex_h * tex_w;
    if (tab.th != tex_h || tab.tw != tex_w) {
        HC_TRY(tab.faces.ensure(sizeof(int) * (size_t)nt));
        HC_TRY(tab.table.ensure(sizeof(float4) * (size_t)nt));
        HC_CUDA(cudaMemsetAsync(tab.faces.ptr, 0xff, sizeof(int) * (size_t)nt, s));
        k_texel_faces<<<div_up(F, 128), 128, 0, s>>>(F, tex_w, tex_h, topo.texcoords.as<float>(), tab.faces.as<int>());
        HC_CHECK_LAUNCH();
        k_texel_table<<<div_up(nt, 256), 256, 0, s>>>(tex_w, tex_h, topo.texcoords.as<float>(), tab.faces.as<int>(),
                                                      tab.table.as<float4>());
        HC_CHECK_LAUNCH();
        tab.th = tex_h;
        tab.tw = tex_w;
    }
    k_uv_map<<<div_up((long long)B * nt, 256), 256, 0, s>>>(B, C, N, nt, mode, topo.faces.as<int3>(),
                                                            tab.table.as<float4>(), verts, vnormal, uv_map);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

}  // namespace hc
