// Test-only harness around the reference embedded-graph kernels.
//
// Part of the parity oracle, not of the product: compiled with the
// UNMODIFIED reference sources CustomTensorFlowCPPOperators/src/
// CustomGPUOperators/EmbeddedGraphOperator/EmbeddedGraphGPUOp{,Grad}.cu into
// oracle/_ref/libhcref.so.  Fills EmbeddedGraphGPUOpData / ...GradData
// (EmbeddedGraphGPUOpData.h:23-62, EmbeddedGraphGPUOpGradData.h) from plain
// arrays instead of the character / graph files and calls the reference's
// extern "C" launchers.  All pointers are device pointers.
#include <cuda_runtime.h>
#include <string.h>

#include "EmbeddedGraphGPUOpData.h"
#include "EmbeddedGraphGPUOpGradData.h"

extern "C" void computeEmbeddedGraphGPUOpGPU(EmbeddedGraphGPUOpData& data);
extern "C" void computeEmbeddedGraphGPUOpGradGPU(EmbeddedGraphGPUOpGradData& data);

extern "C" int hcref_eg_forward(int B, int N, int M, int Mk, int F, const float* base, const int* faces,
                                const int* vf, const int* vf_id, const int* node_vertex, const int* v2n_off,
                                const int* v2n_size, const int* v2n_idx, const float* v2n_w, const int* m2n,
                                const float* markers, const float* dT, const float* dA, const float* sT,
                                const float* sA, const float* disp, float* out_v, float* out_n, float* out_m,
                                float* out_g, float* out_da, float* out_sa) {
    EmbeddedGraphGPUOpData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfNodes = M;
    d.numberOfVertices = N;
    d.numberOfMarkers = Mk;
    d.d_EGVertexToNodeSizes = (int*)v2n_size;
    d.d_EGVertexToNodeIndices = (int*)v2n_idx;
    d.d_EGVertexToNodeOffsets = (int*)v2n_off;
    d.d_EGVertexToNodeWeights = (float*)v2n_w;
    d.d_EGNodeToBaseMeshVertices = (int*)node_vertex;
    d.d_EGMarkerToNodeMapping = (int*)m2n;
    d.d_baseVertices = (float3*)base;
    d.d_baseNormals = nullptr;
    d.d_baseMarkers = (float3*)markers;
    d.d_facesVertex = (int3*)faces;
    d.d_vertexFaces = (int*)vf;
    d.d_vertexFacesId = (int2*)vf_id;
    d.F = F;
    d.d_deltaT = dT;
    d.d_deltaA = dA;
    d.d_skinnedT = sT;
    d.d_skinnedA = sA;
    d.d_displacements = disp;
    d.d_deformedVertices = out_v;
    d.d_deformedNormals = out_n;
    d.d_deformedMarkers = out_m;
    d.d_deformedGraph = out_g;
    d.d_nodesDeltaRotation = out_da;
    d.d_nodesSkinnedRotation = out_sa;
    computeEmbeddedGraphGPUOpGPU(d);
    return (int)cudaDeviceSynchronize();
}

extern "C" int hcref_eg_backward(int B, int N, int M, int Mk, const float* base, const int* node_vertex,
                                 const int* v2n_off, const int* v2n_size, const int* v2n_idx, const float* v2n_w,
                                 const int* n2v_off, const int* n2v_size, const int* n2v_idx, const float* n2v_w,
                                 const int* n2m, const float* markers, const float* gv, const float* gm,
                                 const float* dA, const float* sA, float* gT, float* gA, float* gsT, float* gsA,
                                 float* gdisp) {
    EmbeddedGraphGPUOpGradData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfVertices = N;
    d.numberOfNodes = M;
    d.numberOfMarkers = Mk;
    d.d_EGNodeToVertexSizes = (int*)n2v_size;
    d.d_EGNodeToVertexOffsets = (int*)n2v_off;
    d.d_EGNodeToVertexIndices = (int*)n2v_idx;
    d.d_EGNodeToVertexWeights = (float*)n2v_w;
    d.d_EGVertexToNodeSizes = (int*)v2n_size;
    d.d_EGVertexToNodeIndices = (int*)v2n_idx;
    d.d_EGVertexToNodeOffsets = (int*)v2n_off;
    d.d_EGVertexToNodeWeights = (float*)v2n_w;
    d.d_EGNodeToBaseMeshVertices = (int*)node_vertex;
    d.d_EGNodeToMarkerMapping = (int*)n2m;
    d.d_baseVertices = (float3*)base;
    d.d_baseMarkers = (float3*)markers;
    d.d_inputDeformedVerticesGrad = gv;
    d.d_inputDeformedMarkersGrad = gm;
    d.d_inputDeltaA = dA;
    d.d_inputSkinnedA = sA;
    d.d_outputNodeTGrad = gT;
    d.d_outputNodeRGrad = gA;
    d.d_outputNodeSkinnedTGrad = gsT;
    d.d_outputNodeSkinnedRGrad = gsA;
    d.d_displacementsGrad = gdisp;
    computeEmbeddedGraphGPUOpGradGPU(d);
    return (int)cudaDeviceSynchronize();
}
