// Test-only harness around the reference embedded-graph ARAP kernels.
//
// Part of the parity oracle, not of the product: compiled with the
// UNMODIFIED reference sources CustomTensorFlowCPPOperators/src/
// CustomGPUOperators/EmbeddedGraphARAPOperator/EmbeddedGraphArapGPUOp{,Grad}.cu
// into oracle/_ref/libhcref.so.  Fills EmbeddedGraphArapGPUOpData /
// ...GradData (EmbeddedGraphArapGPUOpData.h:23-47,
// EmbeddedGraphArapGPUOpGradData.h:23-45) from plain arrays instead of the
// character / graph files and calls the reference's extern "C" launchers.
// All pointers are device pointers.
#include <cuda_runtime.h>
#include <string.h>

#include "EmbeddedGraphArapGPUOpData.h"
#include "EmbeddedGraphArapGPUOpGradData.h"

extern "C" void computeEmbeddedGraphArapGPUOpGPU(EmbeddedGraphArapGPUOpData& data);
extern "C" void computeEmbeddedGraphArapGPUOpGradGPU(EmbeddedGraphArapGPUOpGradData& data);

extern "C" int hcref_arap_forward(int B, int M, int maxc, const int* n2n_size, const int* n2n_idx,
                                  const int* n2n_off, const float* rigidity, const int* node_vertex,
                                  const float* base, const float* T, const float* A, float* loss, float* weights,
                                  float* rotation) {
    EmbeddedGraphArapGPUOpData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfNodes = M;
    d.maxNumberOfNodeConnections = maxc;
    d.d_EGNodeToNodeSizes = (int*)n2n_size;
    d.d_EGNodeToNodeIndices = (int*)n2n_idx;
    d.d_EGNodeToNodeOffsets = (int*)n2n_off;
    d.d_EGNodeRigidityWeights = (float*)rigidity;
    d.d_EGNodeToBaseMeshVertices = (int*)node_vertex;
    d.d_baseVertices = (float3*)base;
    d.d_T = T;
    d.d_A = A;
    d.d_nodesArapLoss = loss;
    d.d_connectionWeights = weights;
    d.d_rotation = rotation;
    computeEmbeddedGraphArapGPUOpGPU(d);
    return (int)cudaDeviceSynchronize();
}

extern "C" int hcref_arap_backward(int B, int M, int maxc, const int* n2n_size, const int* n2n_idx,
                                   const int* n2n_off, const float* rigidity, const int* node_vertex,
                                   const float* base, const float* gloss, const float* A, float* gT, float* gA) {
    EmbeddedGraphArapGPUOpGradData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfNodes = M;
    d.maxNumberOfNodeConnections = maxc;
    d.d_EGNodeToNodeSizes = (int*)n2n_size;
    d.d_EGNodeToNodeIndices = (int*)n2n_idx;
    d.d_EGNodeToNodeOffsets = (int*)n2n_off;
    d.d_EGNodeRigidityWeights = (float*)rigidity;
    d.d_EGNodeToBaseMeshVertices = (int*)node_vertex;
    d.d_baseVertices = (float3*)base;
    d.d_nodeArapLossGrad = gloss;
    d.d_A = A;
    d.d_T_grad = gT;
    d.d_A_grad = gA;
    computeEmbeddedGraphArapGPUOpGradGPU(d);
    return (int)cudaDeviceSynchronize();
}
