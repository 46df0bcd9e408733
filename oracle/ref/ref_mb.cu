// Test-only harness around the reference ProjectedMeshBoundaryGpu kernels.
//
// Part of the parity oracle, not of the product: compiled with the
// UNMODIFIED reference source CustomTensorFlowCPPOperators/src/Skeletool/
// Mesh/CUDABasedRasterization.cu into oracle/_ref/libhcref_mb.so (a library
// of its own: that file's renderBuffersGPU has the same C name as the
// renderer's).  Fills the reference's input struct the way the op does
// (ProjectedMeshBoundaryGPUOp.cpp:139-160, CUDABasedRasterization.cpp) and
// calls its extern "C" launchers; all pointers are device pointers.
#include <cuda_runtime.h>
#include <string.h>

#include "CUDABasedRasterizationInput.h"

extern "C" void renderBuffersGPU(CUDABasedRasterizationInput& input, bool usePreviousDisplacement);
extern "C" void checkVisibilityGPU(CUDABasedRasterizationInput& input, bool checkBoundary,
                                   bool useGapDetectionForBoundary);

// Scratch that the op allocates once in its constructor (bounding boxes,
// projected vertices, coverage); kept across calls here too, grown on demand.
static void* g_scratch[3] = {nullptr, nullptr, nullptr};
static size_t g_bytes[3] = {0, 0, 0};

static cudaError_t scratch(int k, size_t bytes, void** out) {
    if (bytes > g_bytes[k]) {
        cudaFree(g_scratch[k]);
        g_scratch[k] = nullptr;
        g_bytes[k] = 0;
        cudaError_t e = cudaMalloc(&g_scratch[k], bytes);
        if (e != cudaSuccess) return e;
        g_bytes[k] = bytes;
    }
    *out = g_scratch[k];
    return cudaSuccess;
}

// faces int32 [F,3]; points [B,N,3]; extr [B,12C]; intr [B,9C]; out bool [B,C,N].
extern "C" int hcref_mesh_boundary(int B, int C, int N, int F, int W, int H, const int* faces, const float* pts,
                                   const float* extr, const float* intr, unsigned char* out) {
    CUDABasedRasterizationInput in;
    memset(&in, 0, sizeof(in));
    in.F = F;
    in.N = N;
    in.numberOfBatches = B;
    in.numberOfCameras = C;
    in.w = W;
    in.h = H;
    in.d_facesVertex = (int3*)faces;
    in.d_vertices = (float3*)pts;
    in.d_boundaries = (bool*)out;
    in.d_cameraExtrinsics = (float4*)extr;
    in.d_cameraIntrinsics = (float3*)intr;
    void *bb = nullptr, *pv = nullptr, *db = nullptr;
    cudaError_t e = scratch(0, sizeof(int4) * (size_t)B * C * F, &bb);
    if (e == cudaSuccess) e = scratch(1, sizeof(float3) * (size_t)B * C * N, &pv);
    if (e == cudaSuccess) e = scratch(2, sizeof(bool) * (size_t)B * C * W * H, &db);
    if (e != cudaSuccess) return (int)e;
    in.d_BBoxes = (int4*)bb;
    in.d_projectedVertices = (float3*)pv;
    in.d_depthBuffer = (bool*)db;
    renderBuffersGPU(in, false);
    checkVisibilityGPU(in, true, false);
    return (int)cudaDeviceSynchronize();
}
