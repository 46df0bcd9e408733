// Test-only harness for the reference's UV-space maps (compute_normal_map).
//
// Part of the parity oracle, not of the product: links the UNMODIFIED
// reference host class CudaRenderer/cpp/src/Renderer/CUDABasedRasterization.cpp
// (whose renderBuffers() builds the texel table on the host on the first call,
// :266-330) with its kernels, and drives it per frame the way the TF op does
// (CudaRenderer.cpp:318-343).  All buffers are device pointers.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "CUDABasedRasterization.h"

extern "C" void* hcref_uv_create(int N, const int* faces, int F, const float* texcoords, int C, int W, int H,
                                 const char* albedo, const char* shading, const char* normal_mode) {
    std::vector<int> f(faces, faces + 3 * (size_t)F);
    std::vector<float> t(texcoords, texcoords + 6 * (size_t)F);
    return new CUDABasedRasterization(f, t, N, C, W, H, albedo, shading, normal_mode);
}

// No destroy: the class's destructor frees the camera buffers it was given,
// which belong to the caller (CUDABasedRasterization.cpp:143-144).

extern "C" int hcref_uv_forward(void* h, int B, int N, int C, int W, int H, int TW, int TH, const float* verts,
                                const float* extr, const float* intr, float* bary, int* face, float* render,
                                float* vnormal, float* normal_map) {
    auto* r = static_cast<CUDABasedRasterization*>(h);
    r->setTextureWidth(TW);
    r->setTextureHeight(TH);
    for (int b = 0; b < B; ++b) {
        r->set_D_vertices((float3*)verts + (size_t)b * N);
        r->set_D_extrinsics(extr + (size_t)b * C * 12);
        r->set_D_intrinsics(intr + (size_t)b * C * 9);
        r->set_D_barycentricCoordinatesBuffer(bary + (size_t)b * C * H * W * 2);
        r->set_D_faceIDBuffer(face + (size_t)b * C * H * W);
        r->set_D_renderBuffer(render + (size_t)b * C * H * W * 3);
        r->set_D_vertexNormal((float3*)vnormal + (size_t)b * C * N);
        r->set_D_normalMap((float3*)normal_map + (size_t)b * TW * TH);
        r->renderBuffers();
    }
    return (int)cudaDeviceSynchronize();
}
