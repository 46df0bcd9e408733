// Test-only harness around the reference camera-projection and multi-view
// silhouette-loss kernels.
//
// Part of the parity oracle, not of the product: compiled with the
// UNMODIFIED reference sources CustomTensorFlowCPPOperators/src/
// CustomGPUOperators/{CameraProjectionOperator,MultiViewSilhouetteLossOperator}/*.cu
// into oracle/_ref/libhcref.so.  Fills the reference's data structs and
// calls its extern "C" launchers; all pointers are device pointers.
#include <cuda_runtime.h>
#include <string.h>

#include "CameraProjectionGPUOpData.h"
#include "CameraProjectionGPUOpGradData.h"
#include "MultiViewSilhouetteLossGPUOpData.h"
#include "MultiViewSilhouetteLossGPUOpGradData.h"

extern "C" void computeCameraProjectionGPUOpGPU(CameraProjectionGPUOpData& data, bool isPoint);
extern "C" void computeCameraProjectionGPUOpGradGPU(CameraProjectionGPUOpGradData& data, bool isPoint);
extern "C" void computeMultiViewSilhouetteLossGPUOpGPU(MultiViewSilhouetteLossGPUOpData& data);
extern "C" void computeMultiViewSilhouetteLossGPUOpGradGPU(MultiViewSilhouetteLossGPUOpGradData& data);

extern "C" int hcref_projection_forward(int B, int C, int N, const float* pts, const float* vecs, const float* extr,
                                        const float* intr, int is_point, float* out) {
    CameraProjectionGPUOpData d;
    memset(&d, 0, sizeof(d));
    d.numberOfPoints = N;
    d.numberOfBatches = B;
    d.numberOfCameras = C;
    d.numberOfKernels = B * C * N;
    d.d_cameraExtrinsics = (float4*)extr;
    d.d_cameraIntrinsics = (float3*)intr;
    d.d_inputPointsWorldSpace = pts;
    d.d_inputVectorsWorldSpace = vecs;
    d.d_outputPointsImageSpace = out;
    computeCameraProjectionGPUOpGPU(d, is_point != 0);
    return (int)cudaDeviceSynchronize();
}

extern "C" int hcref_projection_backward(int B, int C, int N, const float* gimg, const float* pts, const float* extr,
                                         const float* intr, int is_point, float* out) {
    CameraProjectionGPUOpGradData d;
    memset(&d, 0, sizeof(d));
    d.numberOfPoints = N;
    d.numberOfBatches = B;
    d.numberOfCameras = C;
    d.numberOfKernels = B * N;
    d.d_cameraExtrinsics = (float4*)extr;
    d.d_cameraIntrinsics = (float3*)intr;
    d.d_inputPointsImageSpace = gimg;
    d.d_inputPointGlobalSpace = pts;
    d.d_outputPointsWorldSpace = out;
    computeCameraProjectionGPUOpGradGPU(d, is_point != 0);
    return (int)cudaDeviceSynchronize();
}

extern "C" int hcref_silhouette_forward(int B, int C, int N, int U, int V, const float* p2d, const float* n2d,
                                        const unsigned char* isb, const unsigned char* dt, const float* crops,
                                        float* res, float* res1, float* dtgrad, float* closest) {
    MultiViewSilhouetteLossGPUOpData d;
    memset(&d, 0, sizeof(d));
    d.frameResolutionU = U;
    d.frameResolutionV = V;
    d.numberOfBatches = B;
    d.numberOfCameras = C;
    d.numberOfPoints = N;
    d.d_inputPointsImageSpace = p2d;
    d.d_inputNormalsImageSpace = n2d;
    d.d_inputIsBoundary = (const bool*)isb;
    d.d_inputDTImage = dt;
    d.d_inputMultiViewCrops = crops;
    d.d_outputMVSilResidual = res;
    d.d_outputMVSilResidual1 = res1;
    d.d_outputDTImageGradients = dtgrad;
    d.d_outputClosestVertexIds = closest;
    computeMultiViewSilhouetteLossGPUOpGPU(d);
    return (int)cudaDeviceSynchronize();
}

extern "C" int hcref_silhouette_backward(int B, int C, int N, int U, int V, const float* g, const float* g1,
                                         const float* dtgrad, const float* closest, const float* crops, float* out) {
    MultiViewSilhouetteLossGPUOpGradData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfCameras = C;
    d.numberOfPoints = N;
    d.frameResolutionU = U;
    d.frameResolutionV = V;
    d.d_inputDTImageGrad = dtgrad;
    d.d_inputDTLossGrad = g;
    d.d_inputDTLossGrad1 = g1;
    d.d_closestVertexId = closest;
    d.d_inputMultiViewCrops = crops;
    d.d_outputPointsImageSpaceGrad = out;
    computeMultiViewSilhouetteLossGPUOpGradGPU(d);
    return (int)cudaDeviceSynchronize();
}
