// Embedded-graph deformation (EmbeddedGraphGpu / EmbeddedGraphGpuGrad).
//
// Reference: CustomTensorFlowCPPOperators/src/CustomGPUOperators/EmbeddedGraphOperator/
// EmbeddedGraphGPUOp.cu:11-240 and EmbeddedGraphGPUOpGrad.cu:9-213, rotations from
// CustomTensorFlowCPPOperators/src/CudaUtils/EmbeddedGraphRotationHelper.h:53-210.
//
//   v_nr = sum_n w_n (R(delta_a_n) (v - g_n) + g_n + delta_t_n) + displacement
//   v'   = sum_s w_s (R(skinned_a_s) v_nr + skinned_t_s)
//
// with R(a) = Rz(a.z) Ry(a.y) Rx(a.x).  The reference re-evaluates both Euler
// rotations (6 sin/cos each) for every (vertex, node) pair; here a node pass
// evaluates them once per (frame, node) into a table the vertex pass gathers
// (1000 nodes x 96 B per frame stays in L1/L2).  The per-vertex arithmetic
// keeps the reference's operation order, so outputs match bit for bit.
//
// Adjoint: the displacement gradient u_v = (sum_s w_s R_s)^T g_v is computed
// once per vertex; node gradients gather u_v over the node -> vertex lists
// (no atomics):  dT_i = sum_v w_i u_v,  dA_i[k] = sum_v w_i (dR_i/da_k (v - g_i)) . u_v.
// In the reference mode the skinned gradients are zero (EmbeddedGraphGPUOpGrad.cu:
// 136-142); the full mode also returns them.
#include <algorithm>
#include <vector>

#include "eg_rot.cuh"
#include "hc_common.cuh"
#include "hc_math.cuh"

namespace hc {
namespace {

__device__ __forceinline__ float3 mtv(const float* M, float3 v) {  // M^T v, M row-major
    return make_float3(M[0] * v.x + M[3] * v.y + M[6] * v.z, M[1] * v.x + M[4] * v.y + M[7] * v.z,
                       M[2] * v.x + M[5] * v.y + M[8] * v.z);
}

// per (frame, node) table: R_delta (9), t_delta (3), R_skinned (9),
// t_skinned (3) and the node's base position g (3), 16-byte aligned so that a
// row of it is one vector load: rows 0-2 hold (R_delta, t_delta), rows 3-5
// (R_skinned, t_skinned), row 6 g
struct __align__(16) NodeRT {
    float rd[9];
    float td[3];
    float rs[9];
    float ts[3];
    float g[3];
    float pad;
};

__global__ void k_eg_nodes(int B, int M, const float* __restrict__ base, const int* __restrict__ node_vertex,
                           const float* __restrict__ dT, const float* __restrict__ dA, const float* __restrict__ sT,
                           const float* __restrict__ sA, NodeRT* __restrict__ tab, float* __restrict__ graph_out,
                           float* __restrict__ dA_copy, float* __restrict__ sA_copy) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * M) return;
    const int n = (int)(i % M);
    const float3 da = ld3(dA + 3 * i), sa = ld3(sA + 3 * i);
    const R33 Rd = euler_rot(da), Rs = euler_rot(sa);
    NodeRT t;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        t.rd[k] = Rd.m[k];
        t.rs[k] = Rs.m[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        t.td[k] = dT[3 * i + k];
        t.ts[k] = sT[3 * i + k];
    }
    const float3 gb = ld3(base + 3LL * node_vertex[n]);
    t.g[0] = gb.x;
    t.g[1] = gb.y;
    t.g[2] = gb.z;
    t.pad = 0.f;
    tab[i] = t;
    if (dA_copy) st3(dA_copy + 3 * i, da);
    if (sA_copy) st3(sA_copy + 3 * i, sa);
    if (graph_out) {
        // deformed graph node (EmbeddedGraphGPUOp.cu:32-44)
        const float3 g = ld3(base + 3LL * node_vertex[n]);
        const float3 vnr = g + ld3(dT + 3 * i);
        const float3 d = mv(Rs, vnr) + ld3(sT + 3 * i);
        st3(graph_out + 3 * i, d);
    }
}

// Deformed vertices (EmbeddedGraphGPUOp.cu:50-125), grid (vertex blocks,
// frames).  The block's vertex -> node entries (a contiguous range of the
// packed CSR) are staged in shared memory by coalesced loads; each (vertex,
// node) pair then reads the node's rotation / translation rows as float4
// loads of the 16-byte aligned table and the vertex as one float4.  Sums in
// the reference's order: v_nr = sum_k w_k (R_dk (v - g_k) + g_k + t_dk) +
// disp, then sum_k w_k (R_sk v_nr + t_sk).
constexpr int kEgBlock = 128;
constexpr int kEgStage = 8 * kEgBlock;  // staged (node, weight) entries per block

__global__ void __launch_bounds__(kEgBlock) k_eg_vertices(int B, int N, int M, const float4* __restrict__ base4,
                                                          const int* __restrict__ poff, const int* __restrict__ pidx,
                                                          const float* __restrict__ pw, const NodeRT* __restrict__ tab,
                                                          const float* __restrict__ disp, float* __restrict__ out,
                                                          float* __restrict__ vnr_out) {
    __shared__ int s_idx[kEgStage];
    __shared__ float s_w[kEgStage];
    const int b = blockIdx.y;
    const int v0 = blockIdx.x * kEgBlock, v1 = min(v0 + kEgBlock, N);
    const int e0 = poff[v0], e1 = poff[v1];
    const bool staged = e1 - e0 <= kEgStage;  // block-uniform
    if (staged)
        for (int e = e0 + (int)threadIdx.x; e < e1; e += kEgBlock) {
            s_idx[e - e0] = pidx[e];
            s_w[e - e0] = pw[e];
        }
    __syncthreads();
    const int v = v0 + (int)threadIdx.x;
    if (v >= N) return;
    const long long i = (long long)b * N + v;
    const int off = poff[v], cnt = poff[v + 1] - off;
    const int* I = staged ? s_idx + (off - e0) : pidx + off;
    const float* Wt = staged ? s_w + (off - e0) : pw + off;
    const float4 vb4 = base4[v];
    const float3 vb = make_float3(vb4.x, vb4.y, vb4.z);
    const float4* T = reinterpret_cast<const float4*>(tab + (long long)b * M);
    constexpr int kRows = sizeof(NodeRT) / sizeof(float4);
    float3 vnr = make_float3(0.f, 0.f, 0.f);
    for (int k = 0; k < cnt; ++k) {
        const float4* q = T + (long long)I[k] * kRows;
        const float w = Wt[k];
        const float4 a = q[0], c = q[1], d = q[2], gg = q[6];
        R33 R;
        R.m[0] = a.x;
        R.m[1] = a.y;
        R.m[2] = a.z;
        R.m[3] = a.w;
        R.m[4] = c.x;
        R.m[5] = c.y;
        R.m[6] = c.z;
        R.m[7] = c.w;
        R.m[8] = d.x;
        const float3 g = make_float3(gg.x, gg.y, gg.z);
        vnr += w * (mv(R, vb - g) + g + make_float3(d.y, d.z, d.w));
    }
    vnr += ld3(disp + 3 * i);
    float3 dsum = make_float3(0.f, 0.f, 0.f);
    for (int k = 0; k < cnt; ++k) {
        const float4* q = T + (long long)I[k] * kRows;
        const float w = Wt[k];
        const float4 a = q[3], c = q[4], d = q[5];
        R33 R;
        R.m[0] = a.x;
        R.m[1] = a.y;
        R.m[2] = a.z;
        R.m[3] = a.w;
        R.m[4] = c.x;
        R.m[5] = c.y;
        R.m[6] = c.z;
        R.m[7] = c.w;
        R.m[8] = d.x;
        dsum += w * (mv(R, vnr) + make_float3(d.y, d.z, d.w));
    }
    st3(out + 3 * i, dsum);
    if (vnr_out) st3(vnr_out + 3 * i, vnr);
}

// normalised area-weighted normal of the deformed mesh (EmbeddedGraphGPUOp.cu:180-225)
__global__ void k_eg_normals(int B, int N, const int3* __restrict__ faces, const int* __restrict__ vf,
                             const int2* __restrict__ vf_id, const float* __restrict__ dv, float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * N) return;
    const int b = (int)(i / N), v = (int)(i % N);
    const float* P = dv + (long long)b * N * 3;
    const int2 r = vf_id[v];
    float3 s = make_float3(0.f, 0.f, 0.f);
    for (int k = r.x; k < r.x + r.y; ++k) {
        const int3 f = faces[vf[k]];
        const float3 v0 = ld3(P + 3 * f.x), v1 = ld3(P + 3 * f.y), v2 = ld3(P + 3 * f.z);
        s += cross(v1 - v0, v2 - v0);
    }
    st3(out + 3 * i, normalize3(s));
}

// deformed markers (EmbeddedGraphGPUOp.cu:129-177)
__global__ void k_eg_markers(int B, int Mk, int M, const float* __restrict__ base, const int* __restrict__ node_vertex,
                             const float* __restrict__ markers, const int* __restrict__ m2n,
                             const NodeRT* __restrict__ tab, float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * Mk) return;
    const int b = (int)(i / Mk), m = (int)(i % Mk);
    const int n = m2n[m];
    const NodeRT& T = tab[(long long)b * M + n];
    const float3 g = ld3(base + 3LL * node_vertex[n]);
    R33 Rd, Rs;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        Rd.m[q] = T.rd[q];
        Rs.m[q] = T.rs[q];
    }
    const float3 mnr = mv(Rd, ld3(markers + 3LL * m) - g) + g + make_float3(T.td[0], T.td[1], T.td[2]);
    st3(out + 3 * i, mv(Rs, mnr) + make_float3(T.ts[0], T.ts[1], T.ts[2]));
}

// ---------------------------------------------------------------------------
// adjoint
// ---------------------------------------------------------------------------

// per (frame, vertex): u_v = (sum_s w_s R_s)^T g_v (= the displacement gradient)
__global__ void k_eg_grad_vertex(int B, int N, int M, const int* __restrict__ v2n_off, const int* __restrict__ v2n_size,
                                 const int* __restrict__ v2n_idx, const float* __restrict__ v2n_w,
                                 const NodeRT* __restrict__ tab, const float* __restrict__ gv,
                                 float* __restrict__ u_out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * N) return;
    const int b = (int)(i / N), v = (int)(i % N);
    const int off = v2n_off[v], cnt = v2n_size[v];
    const NodeRT* T = tab + (long long)b * M;
    float S[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) S[q] = 0.f;
    for (int k = 0; k < cnt; ++k) {
        const int n = v2n_idx[off + k];
        const float w = v2n_w[off + k];
#pragma unroll
        for (int q = 0; q < 9; ++q) S[q] = S[q] + T[n].rs[q] * w;
    }
    st3(u_out + 3 * i, mtv(S, ld3(gv + 3 * i)));
}

// per (frame, node): gather over the node's vertices (and its marker)
__global__ void k_eg_grad_node(int B, int N, int M, int Mk, const float* __restrict__ base,
                               const int* __restrict__ node_vertex, const int* __restrict__ n2v_off,
                               const int* __restrict__ n2v_size, const int* __restrict__ n2v_idx,
                               const float* __restrict__ n2v_w, const int* __restrict__ n2m,
                               const float* __restrict__ markers, const float* __restrict__ dA,
                               const float* __restrict__ sA, const float* __restrict__ gv,
                               const float* __restrict__ gm, const float* __restrict__ u,
                               const float* __restrict__ vnr, const NodeRT* __restrict__ tab, int full,
                               float* __restrict__ gT, float* __restrict__ gA, float* __restrict__ gsT,
                               float* __restrict__ gsA) {
    // one warp per (frame, node): lanes split the node's vertex list, then a
    // warp reduction; lane 0 adds the marker term and writes
    const long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= (long long)B * M) return;  // warp-uniform
    const int b = (int)(i / M), n = (int)(i % M);
    const float3 g = ld3(base + 3LL * node_vertex[n]);
    R33 da, db, dc;
    euler_rot_d(ld3(dA + 3 * i), da, db, dc);
    R33 sda, sdb, sdc;
    if (full) euler_rot_d(ld3(sA + 3 * i), sda, sdb, sdc);
    float3 t = make_float3(0.f, 0.f, 0.f), a = make_float3(0.f, 0.f, 0.f);
    float3 st = make_float3(0.f, 0.f, 0.f), sa = make_float3(0.f, 0.f, 0.f);
    const int off = n2v_off[n], cnt = n2v_size[n];
    for (int k = lane; k < cnt; k += 32) {
        const int v = n2v_idx[off + k];
        const float w = n2v_w[off + k];
        const long long vi = (long long)b * N + v;
        const float3 uv = ld3(u + 3 * vi);
        const float3 d = ld3(base + 3LL * v) - g;
        t += w * uv;
        a += w * make_float3(dot(mv(da, d), uv), dot(mv(db, d), uv), dot(mv(dc, d), uv));
        if (full) {
            const float3 gvv = ld3(gv + 3 * vi), p = ld3(vnr + 3 * vi);
            st += w * gvv;
            sa += w * make_float3(dot(mv(sda, p), gvv), dot(mv(sdb, p), gvv), dot(mv(sdc, p), gvv));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
        t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
        t.z += __shfl_xor_sync(0xffffffffu, t.z, o);
        a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
        a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
        a.z += __shfl_xor_sync(0xffffffffu, a.z, o);
        if (full) {
            st.x += __shfl_xor_sync(0xffffffffu, st.x, o);
            st.y += __shfl_xor_sync(0xffffffffu, st.y, o);
            st.z += __shfl_xor_sync(0xffffffffu, st.z, o);
            sa.x += __shfl_xor_sync(0xffffffffu, sa.x, o);
            sa.y += __shfl_xor_sync(0xffffffffu, sa.y, o);
            sa.z += __shfl_xor_sync(0xffffffffu, sa.z, o);
        }
    }
    if (lane != 0) return;
    const int m = n2m ? n2m[n] : -1;
    if (m >= 0 && gm) {
        // marker residual (EmbeddedGraphGPUOpGrad.cu:90-123): weight 1, its own node
        const NodeRT& T = tab[i];
        const float3 gmm = ld3(gm + 3 * ((long long)b * Mk + m));
        const float3 um = mtv(T.rs, gmm);
        const float3 d = ld3(markers + 3LL * m) - g;
        t += um;
        a += make_float3(dot(mv(da, d), um), dot(mv(db, d), um), dot(mv(dc, d), um));
        if (full) {
            R33 Rd;
#pragma unroll
            for (int q = 0; q < 9; ++q) Rd.m[q] = T.rd[q];
            const float3 p = mv(Rd, d) + g + make_float3(T.td[0], T.td[1], T.td[2]);
            st += gmm;
            sa += make_float3(dot(mv(sda, p), gmm), dot(mv(sdb, p), gmm), dot(mv(sdc, p), gmm));
        }
    }
    st3(gT + 3 * i, t);
    st3(gA + 3 * i, a);
    st3(gsT + 3 * i, st);
    st3(gsA + 3 * i, sa);
}

}  // namespace
}  // namespace hc

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace hc;

struct hc_eg_s {
    int N = 0, M = 0, Mk = 0, F = 0;
    int full_skinned_grad = 0;
    DevBuf base, node_vertex, v2n_off, v2n_size, v2n_idx, v2n_w, n2v_off, n2v_size, n2v_idx, n2v_w;
    DevBuf base4, v2n_poff, v2n_pidx, v2n_pw;  // float4 base vertices; the vertex -> node CSR packed in vertex order
    DevBuf markers, m2n, n2m, faces, vf, vf_id;
    DevBuf tab, u, vnr;
};

namespace hc {
void build_vertex_faces(int N, const int32_t* faces, int F, std::vector<int>& vf, std::vector<int>& vf_id);
}

extern "C" hc_status hc_eg_create(hc_eg* out, int32_t n_vertices, const float* base_vertices, const int32_t* faces,
                                  int32_t n_faces, int32_t n_nodes, const int32_t* node_to_base_vertex,
                                  const int32_t* v2n_offsets, const int32_t* v2n_sizes, const int32_t* v2n_indices,
                                  const float* v2n_weights, const int32_t* n2v_offsets, const int32_t* n2v_sizes,
                                  const int32_t* n2v_indices, const float* n2v_weights, int32_t n_markers,
                                  const float* base_markers, const int32_t* marker_to_node) {
    clear_error();
    HC_REQUIRE(out, "out is NULL");
    *out = nullptr;
    HC_REQUIRE(n_vertices > 0 && n_nodes > 0 && n_faces > 0, "empty mesh or graph");
    HC_REQUIRE(base_vertices && faces && node_to_base_vertex && v2n_offsets && v2n_sizes && v2n_indices &&
                   v2n_weights && n2v_offsets && n2v_sizes && n2v_indices && n2v_weights,
               "NULL graph array");
    HC_REQUIRE(n_markers == 0 || (base_markers && marker_to_node), "markers need positions and node ids");
    long long nv2n = 0, nn2v = 0;
    for (int v = 0; v < n_vertices; ++v) {
        HC_REQUIRE(v2n_sizes[v] >= 0 && v2n_offsets[v] >= 0, "bad vertex->node range at %d", v);
        nv2n = std::max<long long>(nv2n, (long long)v2n_offsets[v] + v2n_sizes[v]);
    }
    for (int n = 0; n < n_nodes; ++n) {
        HC_REQUIRE(n2v_sizes[n] >= 0 && n2v_offsets[n] >= 0, "bad node->vertex range at %d", n);
        HC_REQUIRE(node_to_base_vertex[n] >= 0 && node_to_base_vertex[n] < n_vertices, "node %d vertex out of range",
                   n);
        nn2v = std::max<long long>(nn2v, (long long)n2v_offsets[n] + n2v_sizes[n]);
    }
    for (long long k = 0; k < nv2n; ++k)
        HC_REQUIRE(v2n_indices[k] >= 0 && v2n_indices[k] < n_nodes, "vertex->node index %d out of range",
                   v2n_indices[k]);
    for (long long k = 0; k < nn2v; ++k)
        HC_REQUIRE(n2v_indices[k] >= 0 && n2v_indices[k] < n_vertices, "node->vertex index %d out of range",
                   n2v_indices[k]);
    for (int i = 0; i < 3 * n_faces; ++i)
        HC_REQUIRE(faces[i] >= 0 && faces[i] < n_vertices, "face index out of range");
    std::vector<int> n2m(n_nodes, -1);
    for (int m = 0; m < n_markers; ++m) {
        HC_REQUIRE(marker_to_node[m] >= 0 && marker_to_node[m] < n_nodes, "marker %d node out of range", m);
        n2m[marker_to_node[m]] = m;
    }
    hc_eg_s* h = new hc_eg_s();
    h->N = n_vertices;
    h->M = n_nodes;
    h->Mk = n_markers;
    h->F = n_faces;
    std::vector<int> vf, vf_id;
    build_vertex_faces(n_vertices, faces, n_faces, vf, vf_id);
    hc_status st = HC_OK;
#define UP(buf, ptr, n)                                   \
    if (st == HC_OK) st = upload(h->buf, ptr, (size_t)(n));
    UP(base, base_vertices, 3LL * n_vertices);
    UP(node_vertex, node_to_base_vertex, n_nodes);
    UP(v2n_off, v2n_offsets, n_vertices);
    UP(v2n_size, v2n_sizes, n_vertices);
    UP(v2n_idx, v2n_indices, std::max<long long>(nv2n, 1));
    UP(v2n_w, v2n_weights, std::max<long long>(nv2n, 1));
    UP(n2v_off, n2v_offsets, n_nodes);
    UP(n2v_size, n2v_sizes, n_nodes);
    UP(n2v_idx, n2v_indices, std::max<long long>(nn2v, 1));
    UP(n2v_w, n2v_weights, std::max<long long>(nn2v, 1));
    UP(n2m, n2m.data(), n_nodes);
    UP(faces, faces, 3LL * n_faces);
    UP(vf, vf.data(), vf.size());
    UP(vf_id, vf_id.data(), vf_id.size());
    if (n_markers > 0) {
        UP(markers, base_markers, 3LL * n_markers);
        UP(m2n, marker_to_node, n_markers);
    }
    {
        // the vertex -> node lists packed contiguously in vertex order (the
        // vertex kernel stages a block's range in one coalesced sweep), and
        // the base vertices padded to float4
        std::vector<int> poff((size_t)n_vertices + 1, 0), pidx;
        std::vector<float> pw;
        std::vector<float4> b4((size_t)n_vertices);
        for (int v = 0; v < n_vertices; ++v) {
            for (int k = 0; k < v2n_sizes[v]; ++k) {
                pidx.push_back(v2n_indices[v2n_offsets[v] + k]);
                pw.push_back(v2n_weights[v2n_offsets[v] + k]);
            }
            poff[v + 1] = (int)pidx.size();
            b4[v] = make_float4(base_vertices[3 * v], base_vertices[3 * v + 1], base_vertices[3 * v + 2], 0.f);
        }
        if (pidx.empty()) {
            pidx.push_back(0);
            pw.push_back(0.f);
        }
        UP(v2n_poff, poff.data(), poff.size());
        UP(v2n_pidx, pidx.data(), pidx.size());
        UP(v2n_pw, pw.data(), pw.size());
        UP(base4, b4.data(), b4.size());
    }
#undef UP
    if (st != HC_OK) {
        delete h;
        return st;
    }
    *out = h;
    return HC_OK;
}

extern "C" hc_status hc_eg_destroy(hc_eg h) {
    clear_error();
    if (!h) return HC_OK;
    DevBuf* bufs[] = {&h->base, &h->node_vertex, &h->v2n_off, &h->v2n_size, &h->v2n_idx, &h->v2n_w, &h->n2v_off,
                      &h->n2v_size, &h->n2v_idx, &h->n2v_w, &h->markers, &h->m2n, &h->n2m, &h->faces, &h->vf,
                      &h->vf_id, &h->tab, &h->u, &h->vnr, &h->base4, &h->v2n_poff, &h->v2n_pidx, &h->v2n_pw};
    for (DevBuf* b : bufs) b->release();
    delete h;
    return HC_OK;
}

extern "C" hc_status hc_eg_set_full_skinned_gradient(hc_eg h, int32_t enable) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    h->full_skinned_grad = enable ? 1 : 0;
    return HC_OK;
}

extern "C" hc_status hc_eg_reserve(hc_eg h, int32_t batch) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "invalid handle or batch");
    HC_TRY(h->tab.ensure(sizeof(NodeRT) * (size_t)batch * h->M));
    HC_TRY(h->u.ensure(sizeof(float) * 3 * (size_t)batch * h->N));
    HC_TRY(h->vnr.ensure(sizeof(float) * 3 * (size_t)batch * h->N));
    return HC_OK;
}

extern "C" hc_status hc_eg_forward(hc_eg h, void* stream, int32_t batch, const float* nodes_delta_translation,
                                   const float* nodes_delta_rotation, const float* nodes_skinned_translation,
                                   const float* nodes_skinned_rotation, const float* vertex_displacements,
                                   float* deformed_vertices, float* deformed_normals, float* deformed_markers,
                                   float* deformed_graph, float* d_delta_rotation, float* d_skinned_rotation) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(batch > 0, "batch must be positive");
    HC_REQUIRE(nodes_delta_translation && nodes_delta_rotation && nodes_skinned_translation &&
                   nodes_skinned_rotation && vertex_displacements && deformed_vertices,
               "NULL input/output pointer");
    HC_REQUIRE(h->Mk == 0 || deformed_markers, "deformed_markers output missing");
    cudaStream_t s = (cudaStream_t)stream;
    HC_TRY(h->tab.ensure(sizeof(NodeRT) * (size_t)batch * h->M));
    NodeRT* tab = h->tab.as<NodeRT>();
    const long long BM = (long long)batch * h->M, BN = (long long)batch * h->N;
    k_eg_nodes<<<div_up(BM, 128), 128, 0, s>>>(batch, h->M, h->base.as<float>(), h->node_vertex.as<int>(),
                                               nodes_delta_translation, nodes_delta_rotation,
                                               nodes_skinned_translation, nodes_skinned_rotation, tab, deformed_graph,
                                               d_delta_rotation, d_skinned_rotation);
    HC_CHECK_LAUNCH();
    HC_REQUIRE(batch <= 65535, "too many frames in one call (%d)", batch);
    k_eg_vertices<<<dim3(div_up(h->N, kEgBlock), batch), kEgBlock, 0, s>>>(
        batch, h->N, h->M, h->base4.as<float4>(), h->v2n_poff.as<int>(), h->v2n_pidx.as<int>(),
        h->v2n_pw.as<float>(), tab, vertex_displacements, deformed_vertices, nullptr);
    HC_CHECK_LAUNCH();
    if (deformed_normals) {
        k_eg_normals<<<div_up(BN, 128), 128, 0, s>>>(batch, h->N, h->faces.as<int3>(), h->vf.as<int>(),
                                                     h->vf_id.as<int2>(), deformed_vertices, deformed_normals);
        HC_CHECK_LAUNCH();
    }
    if (h->Mk > 0) {
        k_eg_markers<<<div_up((long long)batch * h->Mk, 128), 128, 0, s>>>(
            batch, h->Mk, h->M, h->base.as<float>(), h->node_vertex.as<int>(), h->markers.as<float>(),
            h->m2n.as<int>(), tab, deformed_markers);
        HC_CHECK_LAUNCH();
    }
    return HC_OK;
}

extern "C" hc_status hc_eg_backward(hc_eg h, void* stream, int32_t batch, const float* deformed_vertices_grad,
                                    const float* deformed_markers_grad, const float* d_delta_a,
                                    const float* d_skinned_a, float* nodes_t_grad, float* nodes_r_grad,
                                    float* nodes_skinned_t_grad, float* nodes_skinned_r_grad,
                                    float* vertex_displacements_grad, const float* nodes_delta_translation,
                                    const float* vertex_displacements) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(batch > 0, "batch must be positive");
    HC_REQUIRE(deformed_vertices_grad && d_delta_a && d_skinned_a && nodes_t_grad && nodes_r_grad &&
                   nodes_skinned_t_grad && nodes_skinned_r_grad && vertex_displacements_grad,
               "NULL input/output pointer");
    const bool full = h->full_skinned_grad != 0;
    HC_REQUIRE(!full || (nodes_delta_translation && vertex_displacements),
               "the full skinned gradient needs nodes_delta_translation and vertex_displacements");
    cudaStream_t s = (cudaStream_t)stream;
    HC_TRY(h->tab.ensure(sizeof(NodeRT) * (size_t)batch * h->M));
    const long long BM = (long long)batch * h->M, BN = (long long)batch * h->N;
    NodeRT* tab = h->tab.as<NodeRT>();
    // node table from the saved angles; the backward reads the rotations, and
    // (full mode) the delta translations -- the skinned-translation slot of
    // the table is unused here, so it is filled from the same array
    k_eg_nodes<<<div_up(BM, 128), 128, 0, s>>>(batch, h->M, h->base.as<float>(), h->node_vertex.as<int>(),
                                               full ? nodes_delta_translation : d_delta_a, d_delta_a,
                                               full ? nodes_delta_translation : d_delta_a, d_skinned_a, tab, nullptr,
                                               nullptr, nullptr);
    HC_CHECK_LAUNCH();
    if (full) {
        HC_TRY(h->vnr.ensure(sizeof(float) * 3 * (size_t)BN));
        HC_TRY(h->u.ensure(sizeof(float) * 3 * (size_t)BN));
        // v_nr of every vertex (the outer sum's argument); the deformed output
        // goes to the scratch u buffer and is overwritten below
        HC_REQUIRE(batch <= 65535, "too many frames in one call (%d)", batch);
        k_eg_vertices<<<dim3(div_up(h->N, kEgBlock), batch), kEgBlock, 0, s>>>(
            batch, h->N, h->M, h->base4.as<float4>(), h->v2n_poff.as<int>(), h->v2n_pidx.as<int>(),
            h->v2n_pw.as<float>(), tab, vertex_displacements, h->u.as<float>(), h->vnr.as<float>());
        HC_CHECK_LAUNCH();
    }
    k_eg_grad_vertex<<<div_up(BN, 128), 128, 0, s>>>(batch, h->N, h->M, h->v2n_off.as<int>(), h->v2n_size.as<int>(),
                                                     h->v2n_idx.as<int>(), h->v2n_w.as<float>(), tab,
                                                     deformed_vertices_grad, vertex_displacements_grad);
    HC_CHECK_LAUNCH();
    k_eg_grad_node<<<div_up(BM * 32, 256), 256, 0, s>>>(
        batch, h->N, h->M, h->Mk, h->base.as<float>(), h->node_vertex.as<int>(), h->n2v_off.as<int>(),
        h->n2v_size.as<int>(), h->n2v_idx.as<int>(), h->n2v_w.as<float>(), h->n2m.as<int>(), h->markers.as<float>(),
        d_delta_a, d_skinned_a, deformed_vertices_grad, deformed_markers_grad, vertex_displacements_grad,
        full ? h->vnr.as<float>() : nullptr, tab, full ? 1 : 0, nodes_t_grad, nodes_r_grad, nodes_skinned_t_grad,
        nodes_skinned_r_grad);
    HC_CHECK_LAUNCH();
    return HC_OK;
}
