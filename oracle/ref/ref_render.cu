// Test-only harness around the reference rasterizer kernels.
//
// This file is part of the parity oracle, not of the product: it is compiled
// together with the UNMODIFIED reference sources
// CudaRenderer/cpp/src/Renderer/CUDABasedRasterization.cu and
// CUDABasedRasterizationGrad.cu (read in place from the reference tree by
// oracle/Makefile) into oracle/_ref/libhcref.so.  It fills the reference's
// input structs (CUDABasedRasterizationInput.h:42-109,
// CUDABasedRasterizationGradInput.h:26-89) the way the TF op does
// (CudaRenderer.cpp:316-345, CudaRendererGrad.cpp:241-274: one launcher call
// per frame) and calls the reference's extern "C" launchers.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "CUDABasedRasterizationGradInput.h"
#include "CUDABasedRasterizationInput.h"

extern "C" void renderBuffersGPU(CUDABasedRasterizationInput& input);
extern "C" void renderBuffersGradGPU(CUDABasedRasterizationGradInput& input);

namespace {

// Same list construction as CUDABasedRasterization::getVertexFaces
// (CUDABasedRasterization.cpp:154-183) for meshes without isolated vertices.
void vertex_faces(int N, const int* faces, int F, std::vector<int>& vf, std::vector<int>& vfid) {
    std::vector<std::vector<int>> lists(N);
    for (int f = 0; f < F; ++f) {
        const int a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
        lists[a].push_back(f);
        if (b != a) lists[b].push_back(f);
        if (c != a && c != b) lists[c].push_back(f);
    }
    vf.clear();
    vfid.clear();
    for (int v = 0; v < N; ++v) {
        vfid.push_back((int)vf.size());
        vfid.push_back((int)lists[v].size());
        vf.insert(vf.end(), lists[v].begin(), lists[v].end());
    }
}

template <class T>
T* dev_copy(const T* h, size_t n) {
    T* d = nullptr;
    if (cudaMalloc(&d, n * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

}  // namespace

struct hcref_renderer {
    int N, F, C, W, H, albedo, shading, normal_mode, ifs, tfs;
    int3* faces;
    int* vf;
    int2* vfid;
    float* texcoords;
    int4* bboxes;
    float3* projected;
    float3* face_normal;
    int* depth;
    float4* inv_ext;
    float4* inv_proj;
};

extern "C" hcref_renderer* hcref_renderer_create(int N, const int* faces, int F, const float* texcoords, int C,
                                                 int W, int H, int albedo, int shading, int normal_mode,
                                                 int image_filter_size, int texture_filter_size) {
    hcref_renderer* r = new hcref_renderer();
    r->N = N;
    r->F = F;
    r->C = C;
    r->W = W;
    r->H = H;
    r->albedo = albedo;
    r->shading = shading;
    r->normal_mode = normal_mode;
    r->ifs = image_filter_size;
    r->tfs = texture_filter_size;
    std::vector<int> vf, vfid;
    vertex_faces(N, faces, F, vf, vfid);
    r->faces = (int3*)dev_copy(faces, (size_t)3 * F);
    r->vf = dev_copy(vf.data(), vf.size());
    r->vfid = (int2*)dev_copy(vfid.data(), vfid.size());
    std::vector<float> tc((size_t)6 * F, 0.f);
    if (texcoords) memcpy(tc.data(), texcoords, sizeof(float) * 6 * F);
    r->texcoords = dev_copy(tc.data(), tc.size());
    cudaMalloc(&r->bboxes, sizeof(int4) * (size_t)F * C);
    cudaMalloc(&r->projected, sizeof(float3) * (size_t)N * C);
    cudaMalloc(&r->face_normal, sizeof(float3) * (size_t)F * C);
    cudaMalloc(&r->depth, sizeof(int) * (size_t)C * H * W);
    cudaMalloc(&r->inv_ext, sizeof(float4) * 4 * C);
    cudaMalloc(&r->inv_proj, sizeof(float4) * 4 * C);
    return r;
}

extern "C" void hcref_renderer_destroy(hcref_renderer* r) {
    if (!r) return;
    cudaFree(r->faces);
    cudaFree(r->vf);
    cudaFree(r->vfid);
    cudaFree(r->texcoords);
    cudaFree(r->bboxes);
    cudaFree(r->projected);
    cudaFree(r->face_normal);
    cudaFree(r->depth);
    cudaFree(r->inv_ext);
    cudaFree(r->inv_proj);
    delete r;
}

// Forward for B frames; optional outputs: depth [B,C,H,W] int, inverse camera
// matrices [B,C,2,16] (inv(E), inv(K E)).  Returns a cudaError_t value.
extern "C" int hcref_render_forward(hcref_renderer* r, int B, const float* verts, const float* colors,
                                    const float* texture, int TH, int TW, const float* sh, const float* extr,
                                    const float* intr, float* bary, int* face, float* render, float* vnormal,
                                    float* normal_map, int* depth_out, float* inv_out, int sync_each) {
    for (int b = 0; b < B; ++b) {
        CUDABasedRasterizationInput in;
        memset(&in, 0, sizeof(in));
        in.numberOfCameras = r->C;
        in.w = r->W;
        in.h = r->H;
        in.F = r->F;
        in.N = r->N;
        in.d_facesVertex = r->faces;
        in.d_vertexFaces = r->vf;
        in.d_vertexFacesId = r->vfid;
        in.d_textureCoordinates = r->texcoords;
        in.d_textureMapIds = nullptr;
        in.computeNormal = (NormalMode)r->normal_mode;
        in.d_BBoxes = r->bboxes;
        in.d_projectedVertices = r->projected;
        in.d_faceNormal = r->face_normal;
        in.albedoMode = (AlbedoMode)r->albedo;
        in.shadingMode = (ShadingMode)r->shading;
        in.d_inverseExtrinsics = r->inv_ext;
        in.d_inverseProjection = r->inv_proj;
        in.d_vertices = (float3*)verts + (size_t)b * r->N;
        in.d_vertexColor = colors ? (float3*)colors + (size_t)b * r->N : nullptr;
        in.texWidth = TW;
        in.texHeight = TH;
        in.d_textureMap = texture ? texture + (size_t)b * TH * TW * 3 : nullptr;
        in.d_shCoeff = sh ? sh + (size_t)b * r->C * 27 : nullptr;
        in.d_cameraExtrinsics = (float4*)(extr + (size_t)b * r->C * 12);
        in.d_cameraIntrinsics = (float3*)(intr + (size_t)b * r->C * 9);
        in.d_faceIDBuffer = face + (size_t)b * r->C * r->H * r->W;
        in.d_depthBuffer = r->depth;
        in.d_barycentricCoordinatesBuffer = bary + (size_t)b * r->C * r->H * r->W * 2;
        in.d_renderBuffer = render + (size_t)b * r->C * r->H * r->W * 3;
        in.d_vertexNormal = (float3*)vnormal + (size_t)b * r->C * r->N;
        in.d_normalMap = normal_map ? (float3*)normal_map + (size_t)b * TH * TW : nullptr;
        renderBuffersGPU(in);
        if (depth_out)
            cudaMemcpy(depth_out + (size_t)b * r->C * r->H * r->W, r->depth, sizeof(int) * (size_t)r->C * r->H * r->W,
                       cudaMemcpyDeviceToDevice);
        if (inv_out) {
            for (int c = 0; c < r->C; ++c) {
                cudaMemcpy(inv_out + ((size_t)b * r->C + c) * 32, r->inv_ext + 4 * c, sizeof(float4) * 4,
                           cudaMemcpyDeviceToDevice);
                cudaMemcpy(inv_out + ((size_t)b * r->C + c) * 32 + 16, r->inv_proj + 4 * c, sizeof(float4) * 4,
                           cudaMemcpyDeviceToDevice);
            }
        }
        if (sync_each) {
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return (int)e;
        }
    }
    return (int)cudaDeviceSynchronize();
}

// Backward for B frames (renderBuffersGradGPU per frame, CudaRendererGrad.cpp:241-274).
extern "C" int hcref_render_backward(hcref_renderer* r, int B, const float* render_grad, const float* verts,
                                     const float* colors, const float* texture, int TH, int TW, const float* sh,
                                     const float* target, const float* vnormal, const float* bary, const int* face,
                                     const float* extr, const float* intr, float* vpos_grad, float* vcol_grad,
                                     float* tex_grad, float* sh_grad) {
    for (int b = 0; b < B; ++b) {
        CUDABasedRasterizationGradInput in;
        memset(&in, 0, sizeof(in));
        in.numberOfCameras = r->C;
        in.w = r->W;
        in.h = r->H;
        in.F = r->F;
        in.N = r->N;
        in.d_facesVertex = r->faces;
        in.d_textureCoordinates = r->texcoords;
        in.d_vertexFaces = r->vf;
        in.d_vertexFacesId = r->vfid;
        in.albedoMode = (AlbedoMode)r->albedo;
        in.shadingMode = (ShadingMode)r->shading;
        in.d_inverseExtrinsics = r->inv_ext;
        in.d_inverseProjection = r->inv_proj;
        in.imageFilterSize = r->ifs;
        in.textureFilterSize = r->tfs;
        const size_t P = (size_t)r->C * r->H * r->W;
        in.d_renderBufferGrad = (float3*)render_grad + (size_t)b * P;
        in.d_targetBufferGrad = nullptr;
        in.d_vertices = (float3*)verts + (size_t)b * r->N;
        in.d_vertexColor = (float3*)colors + (size_t)b * r->N;
        in.d_textureMap = texture + (size_t)b * TH * TW * 3;
        in.d_shCoeff = sh + (size_t)b * r->C * 27;
        in.d_vertexNormal = (float3*)vnormal + (size_t)b * r->C * r->N;
        in.d_barycentricCoordinatesBuffer = (float2*)bary + (size_t)b * P;
        in.d_faceIDBuffer = (int*)face + (size_t)b * P;
        in.d_targetImage = target + (size_t)b * P * 3;
        in.texWidth = TW;
        in.texHeight = TH;
        in.d_cameraExtrinsics = (float4*)(extr + (size_t)b * r->C * 12);
        in.d_cameraIntrinsics = (float3*)(intr + (size_t)b * r->C * 9);
        in.d_vertexPosGrad = (float3*)vpos_grad + (size_t)b * r->N;
        in.d_vertexColorGrad = (float3*)vcol_grad + (size_t)b * r->N;
        in.d_textureGrad = (float3*)tex_grad + (size_t)b * TH * TW;
        in.d_shCoeffGrad = sh_grad + (size_t)b * r->C * 27;
        renderBuffersGradGPU(in);
    }
    return (int)cudaDeviceSynchronize();
}
