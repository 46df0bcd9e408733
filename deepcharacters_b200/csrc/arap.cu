// As-rigid-as-possible regulariser of the embedded graph (EmbeddedGraphArapGpu /
// EmbeddedGraphArapGpuGrad).
//
// Reference: CustomTensorFlowCPPOperators/src/CustomGPUOperators/
// EmbeddedGraphARAPOperator/EmbeddedGraphArapGPUOp.cu:10-97 (forward) and
// EmbeddedGraphArapGPUOpGrad.cu:9-104 (adjoint); node neighbours and rigidity
// weights from Skeletool/Mesh/EmbeddedGraph.cpp:155-167, 327-436, 460-490.
//
// For node j, neighbour slot s < size_j with neighbour k:
//   r_js = R(a_j) (g_k - g_j) + g_j + t_j - (g_k + t_k),   w_js = (rho_j + rho_k) / 2
// (g = base vertex of the node, rho = rigidity weight); padding slots
// s >= size_j hold zeros.  Outputs [B, nodes, max_connections, 3] and
// [B, nodes, max_connections], plus the rotation input copied for the adjoint.
//
// Adjoint (the reference's, including its choices):
//   dT_j = sum_s (rbar_js - rbar_{k s'})   where s' is the slot of j in k's list
//                                          (the last such slot; 0 if j is not there)
//   dA_j[c] = sum_s (dR/da_c (g_k - g_j)) . rbar_js
// The reference searches k's list for j inside the adjoint, per call; here the
// slot s' is found once when the handle is created.
#include <algorithm>
#include <vector>

#include "eg_rot.cuh"
#include "hc_common.cuh"
#include "hc_math.cuh"

namespace hc {
namespace {

struct ArapGraph {
    int M, maxc;
    const int* off;       // [M] first slot of each node's neighbour list
    const int* size;      // [M]
    const int* idx;       // [sum size] neighbour node ids
    const int* rev;       // [sum size] slot of the node in its neighbour's list, -1 if absent
    const float* rigid;   // [M]
    const int* node_vertex;
    const float* base;    // [N,3]
};

__device__ __forceinline__ float3 node_base(const ArapGraph& G, int n) {
    const float* p = G.base + 3LL * G.node_vertex[n];
    return make_float3(p[0], p[1], p[2]);
}

// one thread per (frame, node, slot), the reference's work split
__global__ void k_arap_forward(int B, ArapGraph G, const float* __restrict__ T, const float* __restrict__ A,
                               float* __restrict__ loss, float* __restrict__ weights, float* __restrict__ rotation) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * G.M * G.maxc) return;
    const int s = (int)(i % G.maxc);
    const long long bn = i / G.maxc;  // frame * M + node
    const int j = (int)(bn % G.M);
    const int b = (int)(bn / G.M);
    const float3 a = make_float3(A[3 * bn], A[3 * bn + 1], A[3 * bn + 2]);
    if (s == 0) {
        rotation[3 * bn] = a.x;
        rotation[3 * bn + 1] = a.y;
        rotation[3 * bn + 2] = a.z;
    }
    float3 r = make_float3(0.f, 0.f, 0.f);
    float w = 0.f;
    if (s < G.size[j]) {
        const int k = G.idx[G.off[j] + s];
        const long long bk = (long long)b * G.M + k;
        const float3 tj = make_float3(T[3 * bn], T[3 * bn + 1], T[3 * bn + 2]);
        const float3 tk = make_float3(T[3 * bk], T[3 * bk + 1], T[3 * bk + 2]);
        const float3 gj = node_base(G, j), gk = node_base(G, k);
        r = mv(euler_rot(a), gk - gj) + gj + tj - (gk + tk);
        w = (G.rigid[j] + G.rigid[k]) / 2.f;
    }
    loss[3 * i] = r.x;
    loss[3 * i + 1] = r.y;
    loss[3 * i + 2] = r.z;
    weights[i] = w;
}

// one thread per (frame, node): its slots' residual gradients, and for dT the
// reverse slots of its neighbours (a gather: no atomics)
__global__ void k_arap_backward(int B, ArapGraph G, const float* __restrict__ gloss, const float* __restrict__ A,
                                float* __restrict__ gT, float* __restrict__ gA) {
    const long long bn = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (bn >= (long long)B * G.M) return;
    const int j = (int)(bn % G.M);
    const int b = (int)(bn / G.M);
    R33 da, db, dc;
    euler_rot_d(make_float3(A[3 * bn], A[3 * bn + 1], A[3 * bn + 2]), da, db, dc);
    const float3 gj = node_base(G, j);
    float3 sT = make_float3(0.f, 0.f, 0.f), sA = make_float3(0.f, 0.f, 0.f);
    const int n = G.size[j], o = G.off[j];
    for (int s = 0; s < n; ++s) {
        const int k = G.idx[o + s];
        const float* g = gloss + 3 * (bn * G.maxc + s);
        const float3 rjs = make_float3(g[0], g[1], g[2]);
        const float3 d = node_base(G, k) - gj;
        // columns dR/da_c d, contracted with rbar (the transposed product)
        const float3 ca = mv(da, d), cb = mv(db, d), cc = mv(dc, d);
        sA += make_float3(ca.x * rjs.x + ca.y * rjs.y + ca.z * rjs.z, cb.x * rjs.x + cb.y * rjs.y + cb.z * rjs.z,
                          cc.x * rjs.x + cc.y * rjs.y + cc.z * rjs.z);
        float3 rks = make_float3(0.f, 0.f, 0.f);
        const int sr = G.rev[o + s];
        if (sr >= 0) {
            const float* h = gloss + 3 * (((long long)b * G.M + k) * G.maxc + sr);
            rks = make_float3(h[0], h[1], h[2]);
        }
        sT += rjs - rks;
    }
    gT[3 * bn] = sT.x;
    gT[3 * bn + 1] = sT.y;
    gT[3 * bn + 2] = sT.z;
    gA[3 * bn] = sA.x;
    gA[3 * bn + 1] = sA.y;
    gA[3 * bn + 2] = sA.z;
}

}  // namespace
}  // namespace hc

using namespace hc;

struct hc_arap_s {
    int N = 0, M = 0, maxc = 0;
    DevBuf base, node_vertex, off, size, idx, rev, rigid;
    ArapGraph graph() const {
        ArapGraph G;
        G.M = M;
        G.maxc = maxc;
        G.off = off.as<int>();
        G.size = size.as<int>();
        G.idx = idx.as<int>();
        G.rev = rev.as<int>();
        G.rigid = rigid.as<float>();
        G.node_vertex = node_vertex.as<int>();
        G.base = base.as<float>();
        return G;
    }
};

extern "C" hc_status hc_arap_create(hc_arap* out, int32_t n_vertices, const float* base_vertices, int32_t n_nodes,
                                    const int32_t* node_to_base_vertex, const int32_t* n2n_offsets,
                                    const int32_t* n2n_sizes, const int32_t* n2n_indices,
                                    const float* rigidity_weights, int32_t max_connections) {
    clear_error();
    HC_REQUIRE(out, "out is NULL");
    *out = nullptr;
    HC_REQUIRE(n_vertices > 0 && n_nodes > 0 && max_connections > 0, "empty mesh or graph");
    HC_REQUIRE(base_vertices && node_to_base_vertex && n2n_offsets && n2n_sizes && n2n_indices && rigidity_weights,
               "NULL graph array");
    long long total = 0;
    for (int n = 0; n < n_nodes; ++n) {
        HC_REQUIRE(n2n_sizes[n] >= 0 && n2n_offsets[n] >= 0, "bad node->node range at %d", n);
        HC_REQUIRE(n2n_sizes[n] <= max_connections, "node %d has %d neighbours, more than max_connections %d", n,
                   n2n_sizes[n], max_connections);
        HC_REQUIRE(node_to_base_vertex[n] >= 0 && node_to_base_vertex[n] < n_vertices, "node %d vertex out of range",
                   n);
        total = std::max<long long>(total, (long long)n2n_offsets[n] + n2n_sizes[n]);
    }
    for (long long k = 0; k < total; ++k)
        HC_REQUIRE(n2n_indices[k] >= 0 && n2n_indices[k] < n_nodes, "node->node index %d out of range",
                   n2n_indices[k]);
    // the slot of node j in the list of each of its neighbours k (the last one
    // when j appears twice, as the reference's search keeps the last match)
    std::vector<int> rev(std::max<long long>(total, 1), -1);
    for (int j = 0; j < n_nodes; ++j)
        for (int s = 0; s < n2n_sizes[j]; ++s) {
            const int k = n2n_indices[n2n_offsets[j] + s];
            for (int q = 0; q < n2n_sizes[k]; ++q)
                if (n2n_indices[n2n_offsets[k] + q] == j) rev[n2n_offsets[j] + s] = q;
        }
    hc_arap_s* h = new hc_arap_s();
    h->N = n_vertices;
    h->M = n_nodes;
    h->maxc = max_connections;
    hc_status st = HC_OK;
    std::vector<int> idx(n2n_indices, n2n_indices + total);
    if (idx.empty()) idx.push_back(0);
#define UP(buf, ptr, n)                                   \
    if (st == HC_OK) st = upload(h->buf, ptr, (size_t)(n));
    UP(base, base_vertices, 3LL * n_vertices);
    UP(node_vertex, node_to_base_vertex, n_nodes);
    UP(off, n2n_offsets, n_nodes);
    UP(size, n2n_sizes, n_nodes);
    UP(idx, idx.data(), idx.size());
    UP(rev, rev.data(), rev.size());
    UP(rigid, rigidity_weights, n_nodes);
#undef UP
    if (st != HC_OK) {
        delete h;
        return st;
    }
    *out = h;
    return HC_OK;
}

extern "C" hc_status hc_arap_destroy(hc_arap h) {
    clear_error();
    if (!h) return HC_OK;
    DevBuf* bufs[] = {&h->base, &h->node_vertex, &h->off, &h->size, &h->idx, &h->rev, &h->rigid};
    for (DevBuf* b : bufs) b->release();
    delete h;
    return HC_OK;
}

extern "C" hc_status hc_arap_forward(hc_arap h, void* stream, int32_t batch, const float* nodes_translation,
                                     const float* nodes_rotation, float* nodes_arap_loss, float* connection_weights,
                                     float* rotation) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "bad handle or batch");
    HC_REQUIRE(nodes_translation && nodes_rotation && nodes_arap_loss && connection_weights && rotation,
               "NULL pointer");
    const long long n = (long long)batch * h->M * h->maxc;
    k_arap_forward<<<div_up(n, 256), 256, 0, (cudaStream_t)stream>>>(batch, h->graph(), nodes_translation,
                                                                     nodes_rotation, nodes_arap_loss,
                                                                     connection_weights, rotation);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_arap_backward(hc_arap h, void* stream, int32_t batch, const float* nodes_arap_loss_grad,
                                      const float* nodes_rotation, float* nodes_translation_grad,
                                      float* nodes_rotation_grad) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "bad handle or batch");
    HC_REQUIRE(nodes_arap_loss_grad && nodes_rotation && nodes_translation_grad && nodes_rotation_grad,
               "NULL pointer");
    const long long n = (long long)batch * h->M;
    k_arap_backward<<<div_up(n, 128), 128, 0, (cudaStream_t)stream>>>(batch, h->graph(), nodes_arap_loss_grad,
                                                                      nodes_rotation, nodes_translation_grad,
                                                                      nodes_rotation_grad);
    HC_CHECK_LAUNCH();
    return HC_OK;
}
