// Test-only harness around the reference DQ / LBS skinning kernels.
//
// Part of the parity oracle, not of the product: compiled with the
// UNMODIFIED reference sources CustomTensorFlowCPPOperators/src/
// CustomGPUOperators/{DQSkinningOperator,LBSkinningOperator}/*.cu into
// oracle/_ref/libhcref.so.  The reference computes the per-joint dual
// quaternions / transforms with Eigen on the host (not buildable here: Eigen
// and the character loaders are absent), so the harness takes them as inputs
// and drives only the reference's GPU kernels.  Two harness choices keep the
// reference kernels inside their buffers:
//  * the per-dof influence list gets one -1 sentinel slot more than the
//    longest list (the reference sizes it to exactly the longest list,
//    DQSkinningGPUOpGrad.cpp:124-140, so its dof loop runs past the end of
//    the longest one);
//  * LBS base vertices / normals are replicated per frame (the reference
//    indexes them with the frame offset, LBSkinningGPUOp.cu:83-84).
#include <cuda_runtime.h>
#include <string.h>

#include <vector>

#include "DQSkinningGPUOpData.h"
#include "DQSkinningGPUOpGradData.h"
#include "LBSkinningGPUOpData.h"
#include "LBSkinningGPUOpGradData.h"

extern "C" void computeDQSkinningGPUOpGPU(DQSkinningGPUOpData& data);
extern "C" void computeDQSkinningGPUOpGradGPU(DQSkinningGPUOpGradData& data);
extern "C" void computeLBSkinningGPUOpGPU(LBSkinningGPUOpData& data);
extern "C" void computeLBSkinningGPUOpGradGPU(LBSkinningGPUOpGradData& data);

namespace {

template <class T>
T* dcopy(const T* h, size_t n) {
    T* d = nullptr;
    cudaMalloc(&d, n * sizeof(T) + 16);
    cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

// skin index table as (numNodes, indexNodes, nodes) (DQSkinningGPUOp.cpp:30-66)
struct SkinTable {
    int *num, *index, *nodes;
    SkinTable(int N, int K, const int* skin_index) {
        std::vector<int> n(N, K), ix(N);
        for (int v = 0; v < N; ++v) ix[v] = v * K;
        num = dcopy(n.data(), N);
        index = dcopy(ix.data(), N);
        nodes = dcopy(skin_index, (size_t)N * K);
    }
    ~SkinTable() {
        cudaFree(num);
        cudaFree(index);
        cudaFree(nodes);
    }
};

// influence list (DQSkinningGPUOpGrad.cpp:91-215), host arrays in
float4* influence(int N, int K, int J, int D, const int* parent, const int* type, const int* dof_off,
                  const int* dof_joint, const int* skin_joint, const int* skin_index, const float* weights,
                  int& max_entries) {
    std::vector<std::vector<float4>> per_dof(D);
    for (int v = 0; v < N; ++v)
        for (int d = 0; d < D; ++d)
            for (int i = 0; i < K; ++i) {
                const int bone = skin_index[v * K + i];
                const float w = weights[v * K + i];
                for (int pr = skin_joint[bone]; pr >= 0; pr = parent[pr]) {
                    bool drives = false;
                    for (int e = dof_off[d]; e < dof_off[d + 1]; ++e) drives |= dof_joint[e] == pr;
                    if (drives) per_dof[d].push_back(make_float4((float)v, (float)type[pr], (float)pr, w));
                }
            }
    max_entries = 0;
    for (auto& l : per_dof) max_entries = std::max(max_entries, (int)l.size());
    max_entries += 1;  // sentinel slot (see the file comment)
    std::vector<float4> h((size_t)D * max_entries, make_float4(-1.f, -1.f, -1.f, -1.f));
    for (int d = 0; d < D; ++d)
        for (size_t e = 0; e < per_dof[d].size(); ++e) h[(size_t)d * max_entries + e] = per_dof[d][e];
    return dcopy(h.data(), h.size());
}

}  // namespace

// dq: device [B,S,8]; weights device [B,N,K]; base arrays host
extern "C" int hcref_dq_forward(int B, int N, int S, int K, int J, int D, const int* skin_index, const float* base_v,
                                const float* base_n, const float* weights, const float* dq, float* out_v,
                                float* out_n, float* out_dq, float* out_w) {
    SkinTable t(N, K, skin_index);
    float3* bv = (float3*)dcopy(base_v, (size_t)3 * N);
    float3* bn = (float3*)dcopy(base_n, (size_t)3 * N);
    DQSkinningGPUOpData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfJoints = J;
    d.numberOfSkinningJoints = S;
    d.numberOfDofs = D;
    d.numberOfVertices = N;
    d.numberOfSkinJointsPerVertex = K;
    d.d_numNodes = t.num;
    d.d_indexNodes = t.index;
    d.d_nodes = t.nodes;
    d.d_baseVertices = bv;
    d.d_baseNormals = bn;
    d.d_inputSkinningWeights = weights;
    d.d_dualQuaternions = (float4*)dq;
    d.d_outputSkinVertices = out_v;
    d.d_outputSkinNormals = out_n;
    d.d_outputDualQuaternions = out_dq;
    d.d_outputSkinningWeights = out_w;
    computeDQSkinningGPUOpGPU(d);
    int e = (int)cudaDeviceSynchronize();
    cudaFree(bv);
    cudaFree(bn);
    return e;
}

extern "C" int hcref_dq_backward(int B, int N, int S, int K, int J, int D, const int* parent, const int* type,
                                 const int* dof_off, const int* dof_joint, const int* skin_joint, const int* skin_index,
                                 const float* file_weights, const float* base_v, const float* gv, const float* vpos,
                                 const float* gpos, const float* gaxis, const float* dq, const float* weights,
                                 float* gdof, float* gw) {
    SkinTable t(N, K, skin_index);
    int maxe = 0;
    float4* infl = influence(N, K, J, D, parent, type, dof_off, dof_joint, skin_joint, skin_index, file_weights, maxe);
    float3* bv = (float3*)dcopy(base_v, (size_t)3 * N);
    DQSkinningGPUOpGradData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfVertices = N;
    d.numberOfDofs = D;
    d.numberOfJoints = J;
    d.numberOfSkinningJoints = S;
    d.numberOfSkinJointsPerVertex = K;
    d.maxEntriesPerDofs = maxe;
    d.d_vertexInfluence = infl;
    d.d_baseVertices = bv;
    d.d_numNodes = t.num;
    d.d_indexNodes = t.index;
    d.d_nodes = t.nodes;
    d.d_inputSkinVerticesGrad = gv;
    d.d_inputSkinVertexPositions = vpos;
    d.d_inputJointGlobalPosition = gpos;
    d.d_inputJointGlobalAxis = gaxis;
    d.d_inputDualQuaternions = dq;
    d.d_inputSkinningWeights = weights;
    d.d_outputDofsGrad = gdof;
    d.d_outputSkinningWeightsGrad = gw;
    computeDQSkinningGPUOpGradGPU(d);
    int e = (int)cudaDeviceSynchronize();
    cudaFree(infl);
    cudaFree(bv);
    return e;
}

// xf12: host [B,S,12] (R row-major, t); weights / disp device
extern "C" int hcref_lbs_forward(int B, int N, int S, int K, int J, int D, const int* skin_index, const float* base_v,
                                 const float* base_n, const float* weights, const float* disp, const float* xf12,
                                 float* out_v, float* out_n, float* out_xf, float* out_w) {
    SkinTable t(N, K, skin_index);
    std::vector<float> bvr((size_t)B * N * 3), bnr((size_t)B * N * 3);
    for (int b = 0; b < B; ++b) {
        memcpy(&bvr[(size_t)b * N * 3], base_v, sizeof(float) * 3 * N);
        memcpy(&bnr[(size_t)b * N * 3], base_n, sizeof(float) * 3 * N);
    }
    float3* bv = (float3*)dcopy(bvr.data(), bvr.size());
    float3* bn = (float3*)dcopy(bnr.data(), bnr.size());
    std::vector<float3x3> rot((size_t)B * S);
    std::vector<float3> tr((size_t)B * S);
    for (size_t i = 0; i < (size_t)B * S; ++i) {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) rot[i](r, c) = xf12[12 * i + 3 * r + c];
        tr[i] = make_float3(xf12[12 * i + 9], xf12[12 * i + 10], xf12[12 * i + 11]);
    }
    float3x3* drot = dcopy(rot.data(), rot.size());
    float3* dtr = dcopy(tr.data(), tr.size());
    LBSkinningGPUOpData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfJoints = J;
    d.numberOfSkinningJoints = S;
    d.numberOfDofs = D;
    d.numberOfVertices = N;
    d.numberOfSkinJointsPerVertex = K;
    d.d_numNodes = t.num;
    d.d_indexNodes = t.index;
    d.d_nodes = t.nodes;
    d.d_baseVertices = bv;
    d.d_baseNormals = bn;
    d.d_inputSkinningWeights = weights;
    d.d_inputDisplacement = disp;
    d.d_rotations = drot;
    d.d_translations = dtr;
    d.d_outputSkinVertices = out_v;
    d.d_outputSkinNormals = out_n;
    d.d_outputTransformation = out_xf;
    d.d_outputSkinningWeights = out_w;
    computeLBSkinningGPUOpGPU(d);
    int e = (int)cudaDeviceSynchronize();
    cudaFree(bv);
    cudaFree(bn);
    cudaFree(drot);
    cudaFree(dtr);
    return e;
}

extern "C" int hcref_lbs_backward(int B, int N, int S, int K, int J, int D, const int* parent, const int* type,
                                  const int* dof_off, const int* dof_joint, const int* skin_joint,
                                  const int* skin_index, const float* file_weights, const float* base_v,
                                  const float* gv, const float* vpos, const float* gpos, const float* gaxis,
                                  const float* xf12, const float* weights, float* gdof, float* gw, float* gdisp) {
    SkinTable t(N, K, skin_index);
    int maxe = 0;
    float4* infl = influence(N, K, J, D, parent, type, dof_off, dof_joint, skin_joint, skin_index, file_weights, maxe);
    float3* bv = (float3*)dcopy(base_v, (size_t)3 * N);
    LBSkinningGPUOpGradData d;
    memset(&d, 0, sizeof(d));
    d.numberOfBatches = B;
    d.numberOfVertices = N;
    d.numberOfDofs = D;
    d.numberOfJoints = J;
    d.numberOfSkinningJoints = S;
    d.numberOfSkinJointsPerVertex = K;
    d.maxEntriesPerDofs = maxe;
    d.d_vertexInfluence = infl;
    d.d_baseVertices = bv;
    d.d_numNodes = t.num;
    d.d_indexNodes = t.index;
    d.d_nodes = t.nodes;
    d.d_inputSkinVerticesGrad = gv;
    d.d_inputSkinVertexPositions = vpos;
    d.d_inputJointGlobalPosition = gpos;
    d.d_inputJointGlobalAxis = gaxis;
    d.d_inputTransformation = xf12;
    d.d_inputSkinningWeights = weights;
    d.d_outputDofsGrad = gdof;
    d.d_outputSkinningWeightsGrad = gw;
    d.d_outputDisplacementGrad = gdisp;
    computeLBSkinningGPUOpGradGPU(d);
    int e = (int)cudaDeviceSynchronize();
    cudaFree(infl);
    cudaFree(bv);
    return e;
}
