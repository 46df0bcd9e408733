// Forward kinematics on the device and dual-quaternion / linear-blend skinning
// (DqSkinningGpu / LbSkinningGpu and their gradient ops).
//
// Reference: CustomTensorFlowCPPOperators/src/CustomGPUOperators/DQSkinningOperator/
// DQSkinningGPUOp{.cpp,.cu,Grad.cpp,Grad.cu}, .../LBSkinningOperator/LBSkinningGPUOp{.cpp,.cu,Grad.cu},
// DQ helpers CudaUtils/DQHelper.h:22-235, FK Skeletool/Character/joint.cpp:36-229,
// dof.cpp:9-17, DualQuaternion.h:53-69.
//
// The reference copies the dofs to the host on every call, runs the Eigen
// kinematic chain there, and copies dual quaternions / joint frames back
// (DQSkinningGPUOp.cpp:351-389) -- a serialising round trip that cannot be
// captured in a CUDA graph.  Here one thread per frame walks the joint list
// (parents precede children) entirely on the device.
//
// The dof gradient of the reference is a per-dof serial loop over an
// influence list of (vertex, bone, weight, joint) entries (DQSkinningGPUOpGrad.cu:
// 145-206) computing sum w_i (axis_j x (v - c_j)) . g_v.  Written per bone
// that is  axis_j . (A_s - c_j x G_s)  with the bone moments
// A_s = sum_v w (v x g_v) and G_s = sum_v w g_v, so a single parallel
// reduction over vertices replaces the serial loops.
#include <math.h>

#include <algorithm>
#include <vector>

#include "hc_common.cuh"
#include "hc_math.cuh"

namespace hc {
namespace {

constexpr int kRevolute = 0, kPrismatic = 1;

struct Xf {  // rigid transform, row-major 3x3 rotation + translation
    float r[9];
    float t[3];
};

__host__ __device__ inline void axis_angle(const float* a, float th, float* R) {
    // Rodrigues: R = c I + s [a]x + (1 - c) a a^T  (Eigen AngleAxis, joint.cpp:144-148)
    const float c = cosf(th), s = sinf(th), C = 1.f - c;
    const float x = a[0], y = a[1], z = a[2];
    R[0] = c + x * x * C;
    R[1] = x * y * C - z * s;
    R[2] = x * z * C + y * s;
    R[3] = y * x * C + z * s;
    R[4] = c + y * y * C;
    R[5] = y * z * C - x * s;
    R[6] = z * x * C - y * s;
    R[7] = z * y * C + x * s;
    R[8] = c + z * z * C;
}

__host__ __device__ inline void xf_mul(const Xf& A, const Xf& B, Xf& O) {
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j)
            O.r[3 * i + j] = A.r[3 * i] * B.r[j] + A.r[3 * i + 1] * B.r[3 + j] + A.r[3 * i + 2] * B.r[6 + j];
        O.t[i] = A.r[3 * i] * B.t[0] + A.r[3 * i + 1] * B.t[1] + A.r[3 * i + 2] * B.t[2] + A.t[i];
    }
}

// quaternion (x, y, z, w) of a rotation matrix (Shepperd's method), normalised
__host__ __device__ inline void mat_to_quat(const float* R, float* q) {
    const float tr = R[0] + R[4] + R[8];
    if (tr > 0.f) {
        float s = sqrtf(tr + 1.f);
        q[3] = 0.5f * s;
        s = 0.5f / s;
        q[0] = (R[7] - R[5]) * s;
        q[1] = (R[2] - R[6]) * s;
        q[2] = (R[3] - R[1]) * s;
    } else {
        int i = 0;
        if (R[4] > R[0]) i = 1;
        if (R[8] > R[3 * i + i]) i = 2;
        const int j = (i + 1) % 3, k = (j + 1) % 3;
        float s = sqrtf(R[3 * i + i] - R[3 * j + j] - R[3 * k + k] + 1.f);
        q[i] = 0.5f * s;
        s = 0.5f / s;
        q[3] = (R[3 * k + j] - R[3 * j + k]) * s;
        q[j] = (R[3 * j + i] + R[3 * i + j]) * s;
        q[k] = (R[3 * k + i] + R[3 * i + k]) * s;
    }
    const float n = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int c = 0; c < 4; ++c) q[c] /= n;
}

struct Skel {
    int J, D, S, K, N;
    const int* parent;
    const int* type;
    const float* offset;   // [J,3]
    const float* axis;     // [J,3] local
    const float* jscale;   // [J]
    const int* dof_off;    // [D+1]
    const int* dof_joint;  // [E]
    const float* dof_w;    // [E]
    const int* skin_joint;  // [S]
    const float* skin_scale;  // [S]
    const float* t0inv;    // [S,12] inverse rest transform (R 9 + t 3)
    const unsigned char* in_chain;  // [S,J]
    const int* skin_idx;   // [N,K] skinning joint per vertex slot
    const float* base_v;   // [N,3]
    const float* base_n;   // [N,3]
    const float4* base_v4;  // [N] the same, padded to float4 (one 16-byte load per vertex)
    const float4* base_n4;  // [N]
};

// Forward kinematics, one CTA per frame: the joint parameters and every
// joint's local transform are formed in parallel in shared memory, one thread
// composes the chain (parents precede children), and the outputs -- joint
// transforms [B,J], global joint positions / axes [B,J,3], skinning
// transforms [B,S] -- are written in parallel.
__global__ void k_fk(Skel sk, int B, const float* __restrict__ dofs, Xf* __restrict__ joints, float* __restrict__ gpos,
                     float* __restrict__ gaxis, Xf* __restrict__ skin_xf, float* __restrict__ params) {
    extern __shared__ float fk_sm[];
    const int b = blockIdx.x;
    const int J4 = (sk.J + 3) & ~3, E = sk.dof_off[sk.D], E4 = (E + 3) & ~3;
    float* P = fk_sm;                                        // [J]
    Xf* Lx = reinterpret_cast<Xf*>(fk_sm + J4);              // [J] local transforms
    Xf* T = Lx + sk.J;                                       // [J] global transforms
    int* par = reinterpret_cast<int*>(T + sk.J);             // [J] parents
    float* prod = reinterpret_cast<float*>(par + J4);        // [E] dof weight * dof value
    int* ent_joint = reinterpret_cast<int*>(prod + E4);      // [E] joint of each dof entry
    // DOF -> joint parameters (dof.cpp:9-17): the products in parallel, then
    // every joint sums its entries in dof order, the reference's order
    for (int d = threadIdx.x; d < sk.D; d += blockDim.x) {
        const float v = dofs[(long long)b * sk.D + d];
        for (int e = sk.dof_off[d]; e < sk.dof_off[d + 1]; ++e) {
            prod[e] = sk.dof_w[e] * v;
            ent_joint[e] = sk.dof_joint[e];
        }
    }
    for (int j = threadIdx.x; j < sk.J; j += blockDim.x) par[j] = sk.parent[j];
    __syncthreads();
    for (int j = threadIdx.x; j < sk.J; j += blockDim.x) {
        float acc = 0.f;
        for (int e = 0; e < E; ++e)
            if (ent_joint[e] == j) acc += prod[e];
        P[j] = acc;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < sk.J; j += blockDim.x) {
        Xf local;
        const float s = sk.jscale[j];
        const float* ax = sk.axis + 3 * j;
        if (sk.type[j] == kRevolute) {
            axis_angle(ax, P[j], local.r);
            for (int c = 0; c < 3; ++c) local.t[c] = sk.offset[3 * j + c] * s;
        } else {
            for (int c = 0; c < 9; ++c) local.r[c] = (c % 4 == 0) ? 1.f : 0.f;
            for (int c = 0; c < 3; ++c) local.t[c] = sk.offset[3 * j + c] * s + ax[c] * P[j];
        }
        Lx[j] = local;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 0; j < sk.J; ++j) {
            const int p = par[j];
            if (p >= 0) xf_mul(T[p], Lx[j], T[j]);
            else T[j] = Lx[j];
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < sk.J; j += blockDim.x) {
        const Xf X = T[j];
        joints[(long long)b * sk.J + j] = X;
        params[(long long)b * sk.J + j] = P[j];
        const float* ax = sk.axis + 3 * j;
        float* gp = gpos + ((long long)b * sk.J + j) * 3;
        float* ga = gaxis + ((long long)b * sk.J + j) * 3;
        for (int c = 0; c < 3; ++c) {
            gp[c] = X.t[c];
            ga[c] = X.r[3 * c] * ax[0] + X.r[3 * c + 1] * ax[1] + X.r[3 * c + 2] * ax[2];
        }
    }
    // skinning transforms J * scale * J0^-1 (DQSkinningGPUOp.cpp:274-306); the
    // rotation part has the uniform scale divided out (Eigen rotation())
    for (int si = threadIdx.x; si < sk.S; si += blockDim.x) {
        Xf A = T[sk.skin_joint[si]];
        const float sc = sk.skin_scale[si];
        Xf I0;
        for (int c = 0; c < 9; ++c) I0.r[c] = sk.t0inv[12 * si + c] * sc;
        for (int c = 0; c < 3; ++c) I0.t[c] = sk.t0inv[12 * si + 9 + c] * sc;
        Xf O;
        xf_mul(A, I0, O);
        for (int c = 0; c < 9; ++c) O.r[c] /= sc;
        skin_xf[(long long)b * sk.S + si] = O;
    }
}

// dual quaternions of the skinning transforms: rotation (x,y,z,w), translation (x,y,z,w)
// (DualQuaternion.h:58-69)
__global__ void k_dq_from_xf(int BS, const Xf* __restrict__ xf, float* __restrict__ dq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BS) return;
    const Xf X = xf[i];
    float q[4];
    mat_to_quat(X.r, q);
    const float* t = X.t;
    float* o = dq + 8LL * i;
    o[0] = q[0];
    o[1] = q[1];
    o[2] = q[2];
    o[3] = q[3];
    o[7] = -0.5f * (t[0] * q[0] + t[1] * q[1] + t[2] * q[2]);
    o[4] = 0.5f * (t[0] * q[3] + t[1] * q[2] - t[2] * q[1]);
    o[5] = 0.5f * (-t[0] * q[2] + t[1] * q[3] + t[2] * q[0]);
    o[6] = 0.5f * (t[0] * q[1] - t[1] * q[0] + t[2] * q[3]);
}

__global__ void k_xf_to_lbs(int BS, const Xf* __restrict__ xf, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BS) return;
    for (int c = 0; c < 9; ++c) out[12LL * i + c] = xf[i].r[c];
    for (int c = 0; c < 3; ++c) out[12LL * i + 9 + c] = xf[i].t[c];
}

__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ float4 f4(const float* p) { return make_float4(p[0], p[1], p[2], p[3]); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 mul4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }

// rotation of a point by a unit quaternion (DQHelper.h:53-72)
__device__ __forceinline__ float3 dq_rot(float4 q, float3 v) {
    const float R00 = 1.f - 2.f * q.y * q.y - 2.f * q.z * q.z;
    const float R01 = 2.f * q.y * q.x - 2.f * q.z * q.w;
    const float R02 = 2.f * q.z * q.x + 2.f * q.y * q.w;
    const float R10 = 2.f * q.y * q.x + 2.f * q.z * q.w;
    const float R11 = 1.f - 2.f * q.x * q.x - 2.f * q.z * q.z;
    const float R12 = 2.f * q.z * q.y - 2.f * q.x * q.w;
    const float R20 = 2.f * q.z * q.x - 2.f * q.y * q.w;
    const float R21 = 2.f * q.z * q.y + 2.f * q.x * q.w;
    const float R22 = 1.f - 2.f * q.x * q.x - 2.f * q.y * q.y;
    return make_float3(R00 * v.x + R01 * v.y + R02 * v.z, R10 * v.x + R11 * v.y + R12 * v.z,
                       R20 * v.x + R21 * v.y + R22 * v.z);
}

// translation of a dual quaternion (DQHelper.h:77-86)
__device__ __forceinline__ float3 dq_trans(float4 r, float4 t) {
    return make_float3(2.0f * (-t.w * r.x + t.x * r.w - t.y * r.z + t.z * r.y),
                       2.0f * (-t.w * r.y + t.x * r.z + t.y * r.w - t.z * r.x),
                       2.0f * (-t.w * r.z - t.x * r.y + t.y * r.x + t.z * r.w));
}

// rotation matrix of a unit quaternion (DQHelper.h:22-48)
__device__ __forceinline__ void dq_rotmat(float4 q, float* R) {
    const float twx = 2.f * q.x * q.w, twy = 2.f * q.y * q.w, twz = 2.f * q.z * q.w;
    const float txx = 2.f * q.x * q.x, txy = 2.f * q.y * q.x, txz = 2.f * q.z * q.x;
    const float tyy = 2.f * q.y * q.y, tyz = 2.f * q.z * q.y, tzz = 2.f * q.z * q.z;
    R[0] = 1.f - tyy - tzz;
    R[1] = txy - twz;
    R[2] = txz + twy;
    R[3] = txy + twz;
    R[4] = 1.f - txx - tzz;
    R[5] = tyz - twx;
    R[6] = txz - twy;
    R[7] = tyz + twx;
    R[8] = 1.f - txx - tyy;
}

// sign-aligned weighted blend of a vertex's dual quaternions (DQSkinningGPUOp.cu:65-92)
__device__ __forceinline__ void dq_blend(const Skel& sk, int b, int v, const float* __restrict__ dq,
                                         const float* __restrict__ w, float4& br, float4& bt) {
    br = make_float4(0.f, 0.f, 0.f, 0.f);
    bt = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 first = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = 0; k < sk.K; ++k) {
        const int s = sk.skin_idx[(long long)v * sk.K + k];
        const float wk = w[((long long)b * sk.N + v) * sk.K + k];
        const float* q = dq + ((long long)b * sk.S + s) * 8;
        const float4 r = f4(q), t = f4(q + 4);
        float sign = 1.0f;
        if (k == 0) first = r;
        if (dot4(first, r) < 0.f && k != 0) sign = -1.0f;
        br = add4(br, mul4(mul4(r, wk), sign));
        bt = add4(bt, mul4(mul4(t, wk), sign));
    }
}

// Shared-memory staging of a skinning block (grid (vertex blocks, frames),
// blockDim.x vertices of one frame): the frame's joint table (`table_floats`
// floats per skinning joint) and the block's K joint indices and weights per
// vertex, copied by coalesced loads (16-byte vectors when `vec`: K a multiple
// of 4 and 16-byte aligned arrays).  Returns the block's first vertex.
__device__ __forceinline__ int stage_skin_block(const Skel& sk, int b, const float* __restrict__ table,
                                                int table_floats, const float* __restrict__ w, int vec,
                                                float* s_tab, float* s_w, int* s_idx) {
    const float* t0 = table + (long long)b * sk.S * table_floats;
    for (int j = threadIdx.x; j < sk.S * table_floats; j += blockDim.x) s_tab[j] = t0[j];
    const int v0 = blockIdx.x * blockDim.x;
    const int n = min((int)blockDim.x, sk.N - v0) * sk.K;
    const int* gi = sk.skin_idx + (long long)v0 * sk.K;
    const float* gw = w + ((long long)b * sk.N + v0) * sk.K;
    if (vec) {
        for (int e = threadIdx.x; e < n / 4; e += blockDim.x) {
            reinterpret_cast<int4*>(s_idx)[e] = reinterpret_cast<const int4*>(gi)[e];
            reinterpret_cast<float4*>(s_w)[e] = reinterpret_cast<const float4*>(gw)[e];
        }
    } else {
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            s_idx[e] = gi[e];
            s_w[e] = gw[e];
        }
    }
    __syncthreads();
    return v0;
}

// dynamic shared memory of a skinning block
__host__ __device__ constexpr size_t skin_block_smem(int S, int table_floats, int K, int threads) {
    return sizeof(float) * ((size_t)S * table_floats + 2 * (size_t)threads * K);
}

constexpr int kSkinBlock = 128;

// DQ skinning (DQSkinningGPUOp.cu:56-120), grid (vertex blocks, frames): the
// frame's joint dual quaternions ([S][8]) and the block's top-K joint
// indices and weights staged in shared memory, the base vertex and normal
// read as one float4 each.  The blend runs the reference's slot loop on the
// staged values: sign-aligned to the first dual quaternion, normalised when
// its norm exceeds 1e-6, the same operations in the same order
// (bit-identical to the reference kernel on the same inputs).
__global__ void __launch_bounds__(kSkinBlock) k_dq_skin(Skel sk, int B, const float* __restrict__ dq,
                                                        const float* __restrict__ w, float* __restrict__ out_v,
                                                        float* __restrict__ out_n, float* __restrict__ w_copy,
                                                        int vec) {
    extern __shared__ float s_dyn[];
    float* s_dq = s_dyn;
    float* s_w = s_dq + sk.S * 8;
    int* s_idx = reinterpret_cast<int*>(s_w + kSkinBlock * sk.K);
    const int b = blockIdx.y;
    const int v0 = stage_skin_block(sk, b, dq, 8, w, vec, s_dq, s_w, s_idx);
    const int v = v0 + (int)threadIdx.x;
    if (v >= sk.N) return;
    const long long i = (long long)b * sk.N + v;
    const int* I = s_idx + threadIdx.x * sk.K;
    const float* Wt = s_w + threadIdx.x * sk.K;
    float4 br = make_float4(0.f, 0.f, 0.f, 0.f), bt = br, first = br;
    for (int k = 0; k < sk.K; ++k) {
        const float* q = s_dq + I[k] * 8;
        const float wk = Wt[k];
        const float4 r = make_float4(q[0], q[1], q[2], q[3]), t = make_float4(q[4], q[5], q[6], q[7]);
        float sign = 1.0f;
        if (k == 0) first = r;
        if (dot4(first, r) < 0.f && k != 0) sign = -1.0f;
        br = add4(br, mul4(mul4(r, wk), sign));
        bt = add4(bt, mul4(mul4(t, wk), sign));
    }
    float scale = 1.f;
    const float len = sqrtf(dot4(br, br));
    if (len > 0.000001f) scale = 1.f / len;
    br = mul4(br, scale);
    bt = mul4(bt, scale);
    const float4 bv = sk.base_v4[v], bn = sk.base_n4[v];
    const float3 p = dq_rot(br, make_float3(bv.x, bv.y, bv.z)) + dq_trans(br, bt);
    float R[9];
    dq_rotmat(br, R);
    const float3 n0 = make_float3(bn.x, bn.y, bn.z);
    const float3 rn = make_float3(R[0] * n0.x + R[1] * n0.y + R[2] * n0.z, R[3] * n0.x + R[4] * n0.y + R[5] * n0.z,
                                  R[6] * n0.x + R[7] * n0.y + R[8] * n0.z);
    const float nr = 1.f / sqrtf(dot(rn, rn));
    st3(out_v + 3 * i, p);
    st3(out_n + 3 * i, rn * nr);
    if (w_copy)
        for (int k = 0; k < sk.K; ++k) w_copy[i * sk.K + k] = Wt[k];
}

// LBS skinning (LBSkinningGPUOp.cu:49-96), grid (vertex blocks, frames): the
// frame's joint transforms ([S][12]: rotation row-major, translation) and the
// block's slots staged as in k_dq_skin; the reference's slot loop in its order.
__global__ void __launch_bounds__(kSkinBlock) k_lbs_skin(Skel sk, int B, const float* __restrict__ xf12,
                                                         const float* __restrict__ w, const float* __restrict__ disp,
                                                         float* __restrict__ out_v, float* __restrict__ out_n,
                                                         float* __restrict__ w_copy, int vec) {
    extern __shared__ float s_dyn[];
    float* s_xf = s_dyn;
    float* s_w = s_xf + sk.S * 12;
    int* s_idx = reinterpret_cast<int*>(s_w + kSkinBlock * sk.K);
    const int b = blockIdx.y;
    const int v0 = stage_skin_block(sk, b, xf12, 12, w, vec, s_xf, s_w, s_idx);
    const int v = v0 + (int)threadIdx.x;
    if (v >= sk.N) return;
    const long long i = (long long)b * sk.N + v;
    const int* I = s_idx + threadIdx.x * sk.K;
    const float* Wt = s_w + threadIdx.x * sk.K;
    float R[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float3 t = make_float3(0.f, 0.f, 0.f);
    for (int k = 0; k < sk.K; ++k) {
        const float wk = Wt[k];
        const float* X = s_xf + I[k] * 12;
        for (int c = 0; c < 9; ++c) R[c] = R[c] + X[c] * wk;
        t = t + make_float3(X[9], X[10], X[11]) * wk;
    }
    // the reference indexes the base mesh with the frame offset
    // (LBSkinningGPUOp.cu:83-84), out of bounds for B > 1; the base mesh is
    // shared by all frames here
    const float4 bv = sk.base_v4[v], bn = sk.base_n4[v];
    const float3 p = make_float3(bv.x, bv.y, bv.z) + ld3(disp + 3 * i);
    const float3 n0 = make_float3(bn.x, bn.y, bn.z);
    const float3 o = make_float3(R[0] * p.x + R[1] * p.y + R[2] * p.z, R[3] * p.x + R[4] * p.y + R[5] * p.z,
                                 R[6] * p.x + R[7] * p.y + R[8] * p.z) + t;
    const float3 on = make_float3(R[0] * n0.x + R[1] * n0.y + R[2] * n0.z, R[3] * n0.x + R[4] * n0.y + R[5] * n0.z,
                                  R[6] * n0.x + R[7] * n0.y + R[8] * n0.z);
    st3(out_v + 3 * i, o);
    st3(out_n + 3 * i, on);
    if (w_copy)
        for (int k = 0; k < sk.K; ++k) w_copy[i * sk.K + k] = Wt[k];
}

// ---------------------------------------------------------------------------
// adjoints
// ---------------------------------------------------------------------------

// per-bone moments A_s = sum w (v x g), G_s = sum w g over the vertices of a
// frame; one CTA covers 256 vertices of one frame (grid.y = frame)
__global__ void k_bone_moments(Skel sk, const float* __restrict__ vpos, const float* __restrict__ gv,
                               const float* __restrict__ w, float* __restrict__ mom) {
    extern __shared__ float s_mom[];  // [S][6]
    const int b = blockIdx.y;
    for (int i = threadIdx.x; i < sk.S * 6; i += blockDim.x) s_mom[i] = 0.f;
    __syncthreads();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < sk.N) {
        const long long vi = (long long)b * sk.N + v;
        const float3 p = ld3(vpos + 3 * vi), g = ld3(gv + 3 * vi);
        const float3 pg = cross(p, g);
        for (int k = 0; k < sk.K; ++k) {
            const int s = sk.skin_idx[(long long)v * sk.K + k];
            const float wk = w[vi * sk.K + k];
            float* m = s_mom + 6 * s;
            atomicAdd(m + 0, wk * pg.x);
            atomicAdd(m + 1, wk * pg.y);
            atomicAdd(m + 2, wk * pg.z);
            atomicAdd(m + 3, wk * g.x);
            atomicAdd(m + 4, wk * g.y);
            atomicAdd(m + 5, wk * g.z);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < sk.S * 6; i += blockDim.x)
        if (s_mom[i] != 0.f) atomicAdd(mom + (long long)b * sk.S * 6 + i, s_mom[i]);
}

// dof gradient from the bone moments: a dof collects, for every joint it
// drives, axis . (A_s - c x G_s) (revolute) or axis . G_s (prismatic) of the
// bones whose kinematic chain contains that joint
__global__ void k_dof_grad(Skel sk, int B, const float* __restrict__ mom, const float* __restrict__ gpos,
                           const float* __restrict__ gaxis, float* __restrict__ gdof) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * sk.D) return;
    const int b = i / sk.D, d = i % sk.D;
    float acc = 0.f;
    for (int e = sk.dof_off[d]; e < sk.dof_off[d + 1]; ++e) {
        const int j = sk.dof_joint[e];
        const float3 ax = ld3(gaxis + ((long long)b * sk.J + j) * 3);
        const float3 c = ld3(gpos + ((long long)b * sk.J + j) * 3);
        for (int s = 0; s < sk.S; ++s) {
            if (!sk.in_chain[s * sk.J + j]) continue;
            const float* m = mom + ((long long)b * sk.S + s) * 6;
            const float3 A = make_float3(m[0], m[1], m[2]), G = make_float3(m[3], m[4], m[5]);
            acc += sk.type[j] == kRevolute ? dot(ax, A - cross(c, G)) : dot(ax, G);
        }
    }
    gdof[i] = acc;
}

// DQ weight gradient (DQSkinningGPUOpGrad.cu:12-141).  `parity` keeps the
// reference's Jacobian of the rotated point (DQHelper.h:121-174, which adds
// vert.z instead of multiplying by it); otherwise the exact Jacobian.
__global__ void k_dq_weight_grad(Skel sk, int B, const float* __restrict__ dq, const float* __restrict__ w,
                                 const float* __restrict__ gv, int parity, float* __restrict__ gw) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)B * sk.N * sk.K) return;
    const int kk = (int)(idx % sk.K);
    const long long vi = idx / sk.K;
    const int b = (int)(vi / sk.N), v = (int)(vi % sk.N);
    float4 br, bt;
    dq_blend(sk, b, v, dq, w, br, bt);
    const int s0 = sk.skin_idx[(long long)v * sk.K];
    const float4 first = f4(dq + ((long long)b * sk.S + s0) * 8);
    float scale = sqrtf(dot4(br, br));
    const float4 ir = br, it = bt;
    bool small = false;
    if (scale < 0.000001f) {
        scale = 1.f;
        small = true;
    }
    br = mul4(br, 1.f / scale);
    bt = mul4(bt, 1.f / scale);
    const int s = sk.skin_idx[(long long)v * sk.K + kk];
    const float* q = dq + ((long long)b * sk.S + s) * 8;
    float4 fr = f4(q), ft = f4(q + 4);
    const float sign = (dot4(first, fr) < 0.f && kk != 0) ? -1.f : 1.f;
    fr = mul4(fr, sign);
    ft = mul4(ft, sign);
    float ds = dot4(mul4(ir, 1.f / scale), fr);
    if (small) ds = 0.f;
    const float s2 = scale * scale;
    fr = mul4(add4(mul4(fr, scale), mul4(ir, -ds)), 1.f / s2);
    ft = mul4(add4(mul4(ft, scale), mul4(it, -ds)), 1.f / s2);
    // d(point)/d(rotation quaternion) and d(translation)/d(dq) applied to (fr, ft)
    const float3 vb = ld3(sk.base_v + 3LL * v);
    const float x = br.x, y = br.y, z = br.z, ww = br.w;
    const float qd[4] = {fr.x, fr.y, fr.z, fr.w};
    // rows of dR/dq entries (R00..R22 w.r.t. x,y,z,w)
    const float dR[9][4] = {{0.f, -4.f * y, -4.f * z, 0.f},      {2.f * y, 2.f * x, -2.f * ww, -2.f * z},
                            {2.f * z, 2.f * ww, 2.f * x, 2.f * y}, {2.f * y, 2.f * x, 2.f * ww, 2.f * z},
                            {-4.f * x, 0.f, -4.f * z, 0.f},      {-2.f * ww, 2.f * z, 2.f * y, -2.f * x},
                            {2.f * z, -2.f * ww, 2.f * x, -2.f * y}, {2.f * ww, 2.f * z, 2.f * y, 2.f * x},
                            {-4.f * x, -4.f * y, 0.f, 0.f}};
    float3 g = make_float3(0.f, 0.f, 0.f);
    float gr[3];
    for (int r = 0; r < 3; ++r) {
        float acc = 0.f;
        for (int c = 0; c < 4; ++c) {
            const float a0 = dR[3 * r + 0][c], a1 = dR[3 * r + 1][c], a2 = dR[3 * r + 2][c];
            const float jac = parity ? (a0 * vb.x + a1 * vb.y + a2 + vb.z) : (a0 * vb.x + a1 * vb.y + a2 * vb.z);
            acc += jac * qd[c];
        }
        gr[r] = acc;
    }
    g = make_float3(gr[0], gr[1], gr[2]);
    // translation: t = 2 (-t.w r.xyz + t.xyz r.w + ...) (DQHelper.h:184-235)
    const float4 tq = bt;
    const float dTr[3][4] = {{-tq.w, tq.z, -tq.y, tq.x}, {-tq.z, -tq.w, tq.x, tq.y}, {tq.y, -tq.x, -tq.w, tq.z}};
    const float dTt[3][4] = {{ww, -z, y, -x}, {z, ww, -x, -y}, {-y, x, ww, -z}};
    const float ftd[4] = {ft.x, ft.y, ft.z, ft.w};
    for (int r = 0; r < 3; ++r) {
        float acc = 0.f;
        for (int c = 0; c < 4; ++c) acc += 2.f * dTr[r][c] * qd[c] + 2.f * dTt[r][c] * ftd[c];
        gr[r] = acc;
    }
    g = g + make_float3(gr[0], gr[1], gr[2]);
    gw[idx] = dot(g, ld3(gv + 3 * vi));
}

// LBS weight / displacement gradients (LBSkinningGPUOpGrad.cu:11-88).  In the
// parity mode the reference's indexing is kept: the weight gradient reads the
// transform of slot k instead of the vertex's k-th bone and ignores the
// displacement; the displacement gradient reads the weights without the frame
// offset, the transform of slot k, and skips weights below 1e-4.
__global__ void k_lbs_weight_grad(Skel sk, int B, const float* __restrict__ xf12, const float* __restrict__ disp,
                                  const float* __restrict__ gv, int parity, float* __restrict__ gw) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)B * sk.N * sk.K) return;
    const int kk = (int)(idx % sk.K);
    const long long vi = idx / sk.K;
    const int b = (int)(vi / sk.N), v = (int)(vi % sk.N);
    const int s = parity ? kk : sk.skin_idx[(long long)v * sk.K + kk];
    const float* X = xf12 + ((long long)b * sk.S + s) * 12;
    float3 p = ld3(sk.base_v + 3LL * v);
    if (!parity) p = p + ld3(disp + 3 * vi);
    const float3 o = make_float3(X[0] * p.x + X[1] * p.y + X[2] * p.z, X[3] * p.x + X[4] * p.y + X[5] * p.z,
                                 X[6] * p.x + X[7] * p.y + X[8] * p.z) + make_float3(X[9], X[10], X[11]);
    gw[idx] = dot(o, ld3(gv + 3 * vi));
}

__global__ void k_lbs_disp_grad(Skel sk, int B, const float* __restrict__ xf12, const float* __restrict__ w,
                                const float* __restrict__ gv, int parity, float* __restrict__ gd) {
    const long long vi = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (vi >= (long long)B * sk.N) return;
    const int b = (int)(vi / sk.N), v = (int)(vi % sk.N);
    float M[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // sum w R^T
    for (int k = 0; k < sk.K; ++k) {
        const float wk = parity ? w[(long long)v * sk.K + k] : w[vi * sk.K + k];
        if (parity && wk < 1e-4f) continue;
        const int s = parity ? k : sk.skin_idx[(long long)v * sk.K + k];
        const float* X = xf12 + ((long long)b * sk.S + s) * 12;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) M[3 * c + r] += X[3 * r + c] * wk;
    }
    const float3 g = ld3(gv + 3 * vi);
    st3(gd + 3 * vi, make_float3(M[0] * g.x + M[1] * g.y + M[2] * g.z, M[3] * g.x + M[4] * g.y + M[5] * g.z,
                                 M[6] * g.x + M[7] * g.y + M[8] * g.z));
}

// Node-level skinning of the embedded graph (Pose2EmbeddedGraphCPUOp.cpp:129-300):
// per (frame, node) the dual quaternions of the node's base vertex are blended
// with the character's skin weights (same sign alignment and normalisation as
// the vertices), turned into (R, t), and R into Z-Y-X Euler angles
// (x = atan2(R21, R22), y = atan2(-R20, sy), z = atan2(R10, R00); singular
// branch for sy < 1e-6).  The reference runs this on the host for every call.
__global__ void k_pose2eg(Skel sk, int B, int M, const int* __restrict__ node_vertex, const float* __restrict__ dq,
                          const float* __restrict__ w, float* __restrict__ out_t, float* __restrict__ out_a) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * M) return;
    const int b = (int)(i / M), n = (int)(i % M);
    const int v = node_vertex[n];
    float4 br = make_float4(0.f, 0.f, 0.f, 0.f), bt = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 first = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = 0; k < sk.K; ++k) {
        const int s = sk.skin_idx[(long long)v * sk.K + k];
        const float wk = w[(long long)v * sk.K + k];
        const float* q = dq + ((long long)b * sk.S + s) * 8;
        const float4 r = f4(q), t = f4(q + 4);
        float sign = 1.0f;
        if (k == 0) first = r;
        else if (dot4(first, r) < 0.0f) sign = -1.0f;
        br = add4(br, mul4(mul4(r, wk), sign));
        bt = add4(bt, mul4(mul4(t, wk), sign));
    }
    float scale = 1.f;
    const float len = sqrtf(dot4(br, br));
    if (len > 0.000001f) scale = 1.f / len;
    br = mul4(br, scale);
    bt = mul4(bt, scale);
    float R[9];
    dq_rotmat(br, R);
    st3(out_t + 3 * i, dq_trans(br, bt));
    const float sy = sqrtf(R[0] * R[0] + R[3] * R[3]);
    float3 e;
    if (!((double)sy < 1e-6)) {
        e = make_float3(atan2f(R[7], R[8]), atan2f(-R[6], sy), atan2f(R[3], R[0]));
    } else {
        e = make_float3(atan2f(-R[5], R[4]), atan2f(-R[6], sy), 0.f);
    }
    st3(out_a + 3 * i, e);
}

// ---------------------------------------------------------------------------
// Adjoint of the node skinning.  The reference registers no gradient for
// Pose2EmbeddedGraphCpu (Pose2EmbeddedGraphCpu.py:55-60), so joint angles do
// not train through the embedded graph there.  This is the exact adjoint of
// the forward above, node by node:
//   Euler angles <- rotation matrix <- blended, normalised rotation
//   quaternion; translation <- (rotation, translation) quaternions;
//   normalisation; weighted, sign-aligned blend of the joints' dual
//   quaternions (the signs are locally constant).
// The per-joint dual-quaternion gradients G_s (8 floats) are summed over the
// nodes of a frame in shared memory.  A joint angle theta_j moves every
// skinning transform below joint j by the world-frame rotation about the
// joint's axis a through its position c, so
//   d r_s / d theta_j = 1/2 (a, 0) x r_s,
//   d t_s / d theta_j = a x (t_s - c),
//   d tq_s / d theta_j = 1/2 (d t_s, 0) x r_s + 1/2 (t_s, 0) x d r_s
// (tq = 1/2 (t, 0) x r, the translation part of the dual quaternion, "x" the
// quaternion product); a prismatic joint translates them along a.
// ---------------------------------------------------------------------------

// quaternion product (x, y, z, w) convention: (p_v, p_w)(q_v, q_w)
__device__ __forceinline__ float4 qmul(float4 p, float4 q) {
    return make_float4(p.w * q.x + q.w * p.x + (p.y * q.z - p.z * q.y),
                       p.w * q.y + q.w * p.y + (p.z * q.x - p.x * q.z),
                       p.w * q.z + q.w * p.z + (p.x * q.y - p.y * q.x),
                       p.w * q.w - (p.x * q.x + p.y * q.y + p.z * q.z));
}

// d loss / d (blended rotation, translation quaternions) of one node
__device__ void pose2eg_node_grad(float4 br, float4 bt, float3 gT, float3 gE, float4& gbr, float4& gbt) {
    float len = sqrtf(dot4(br, br));
    const bool norm = len > 0.000001f;
    const float scale = norm ? 1.f / len : 1.f;
    const float4 q = mul4(br, scale), t = mul4(bt, scale);
    float R[9];
    dq_rotmat(q, R);
    // Euler angles -> rotation matrix entries
    float gR[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float sy2 = R[0] * R[0] + R[3] * R[3];
    const float sy = sqrtf(sy2);
    {   // y = atan2(-R20, sy)
        const float u = -R[6], den = u * u + sy2;
        if (den > 0.f) {
            gR[6] += gE.y * (-sy / den);
            if (sy > 0.f) {
                const float gsy = gE.y * (-u / den);
                gR[0] += gsy * R[0] / sy;
                gR[3] += gsy * R[3] / sy;
            }
        }
    }
    if (!((double)sy < 1e-6)) {
        const float dx = R[7] * R[7] + R[8] * R[8], dz = sy2;
        if (dx > 0.f) {  // x = atan2(R21, R22)
            gR[7] += gE.x * R[8] / dx;
            gR[8] -= gE.x * R[7] / dx;
        }
        if (dz > 0.f) {  // z = atan2(R10, R00)
            gR[3] += gE.z * R[0] / dz;
            gR[0] -= gE.z * R[3] / dz;
        }
    } else {  // x = atan2(-R12, R11), z = 0
        const float dx = R[5] * R[5] + R[4] * R[4];
        if (dx > 0.f) {
            gR[5] -= gE.x * R[4] / dx;
            gR[4] += gE.x * R[5] / dx;
        }
    }
    // rotation matrix of q = (x, y, z, w)
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    float4 gq;
    gq.x = 2.f * (gR[1] * y + gR[2] * z + gR[3] * y - gR[4] * 2.f * x - gR[5] * w + gR[6] * z + gR[7] * w -
                  gR[8] * 2.f * x);
    gq.y = 2.f * (-gR[0] * 2.f * y + gR[1] * x + gR[2] * w + gR[3] * x + gR[5] * z - gR[6] * w + gR[7] * z -
                  gR[8] * 2.f * y);
    gq.z = 2.f * (-gR[0] * 2.f * z - gR[1] * w + gR[2] * x + gR[3] * w - gR[4] * 2.f * z + gR[5] * y + gR[6] * x +
                  gR[7] * y);
    gq.w = 2.f * (-gR[1] * z + gR[2] * y + gR[3] * z - gR[5] * x - gR[6] * y + gR[7] * x);
    // translation T = dq_trans(q, t), bilinear in q and t
    gq.x += 2.f * (-t.w * gT.x - t.z * gT.y + t.y * gT.z);
    gq.y += 2.f * (t.z * gT.x - t.w * gT.y - t.x * gT.z);
    gq.z += 2.f * (-t.y * gT.x + t.x * gT.y - t.w * gT.z);
    gq.w += 2.f * (t.x * gT.x + t.y * gT.y + t.z * gT.z);
    float4 gt;
    gt.x = 2.f * (w * gT.x + z * gT.y - y * gT.z);
    gt.y = 2.f * (-z * gT.x + w * gT.y + x * gT.z);
    gt.z = 2.f * (y * gT.x - x * gT.y + w * gT.z);
    gt.w = 2.f * (-x * gT.x - y * gT.y - z * gT.z);
    if (norm) {  // q = br / |br|, t = bt / |br|
        const float k = (dot4(br, gq) + dot4(bt, gt)) / (len * len * len);
        gbr = add4(mul4(gq, scale), mul4(br, -k));
        gbt = mul4(gt, scale);
    } else {
        gbr = gq;
        gbt = gt;
    }
}

// one CTA per frame: node gradients -> per-joint dual-quaternion gradients in shared memory
__global__ void k_pose2eg_grad_nodes(Skel sk, int M, const int* __restrict__ node_vertex, const float* __restrict__ dq,
                                     const float* __restrict__ w, const float* __restrict__ gT,
                                     const float* __restrict__ gA, float* __restrict__ gdq) {
    // grid (node slices, frames); every warp accumulates into its own [S][8]
    // copy, and the block adds the copies' sum to the frame's gradient
    extern __shared__ float s_g[];  // [warps][S][8]
    const int b = blockIdx.y;
    const int SS = sk.S * 8;
    for (int i = threadIdx.x; i < SS * (int)(blockDim.x >> 5); i += blockDim.x) s_g[i] = 0.f;
    __syncthreads();
    float* s_w = s_g + SS * (threadIdx.x >> 5);
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < M; n += gridDim.x * blockDim.x) {
        const int v = node_vertex[n];
        float4 br = make_float4(0.f, 0.f, 0.f, 0.f), bt = br, first = br;
        float sgn[16];
        for (int k = 0; k < sk.K; ++k) {
            const int s = sk.skin_idx[(long long)v * sk.K + k];
            const float wk = w[(long long)v * sk.K + k];
            const float* q = dq + ((long long)b * sk.S + s) * 8;
            const float4 r = f4(q), t = f4(q + 4);
            float sign = 1.0f;
            if (k == 0) first = r;
            else if (dot4(first, r) < 0.0f) sign = -1.0f;
            if (k < 16) sgn[k] = sign;
            br = add4(br, mul4(mul4(r, wk), sign));
            bt = add4(bt, mul4(mul4(t, wk), sign));
        }
        const long long o = ((long long)b * M + n) * 3;
        float4 gbr, gbt;
        pose2eg_node_grad(br, bt, ld3(gT + o), ld3(gA + o), gbr, gbt);
        for (int k = 0; k < sk.K && k < 16; ++k) {
            const int s = sk.skin_idx[(long long)v * sk.K + k];
            const float c = w[(long long)v * sk.K + k] * sgn[k];
            float* g = s_w + s * 8;
            atomicAdd(g + 0, c * gbr.x);
            atomicAdd(g + 1, c * gbr.y);
            atomicAdd(g + 2, c * gbr.z);
            atomicAdd(g + 3, c * gbr.w);
            atomicAdd(g + 4, c * gbt.x);
            atomicAdd(g + 5, c * gbt.y);
            atomicAdd(g + 6, c * gbt.z);
            atomicAdd(g + 7, c * gbt.w);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < SS; i += blockDim.x) {
        float acc = 0.f;
        for (int wp = 0; wp < (int)(blockDim.x >> 5); ++wp) acc += s_g[wp * SS + i];
        atomicAdd(gdq + (long long)b * SS + i, acc);
    }
}

// per (frame, dof): sum over the dof's joints and the skinning joints below them
__global__ void k_pose2eg_grad_dofs(Skel sk, int B, const float* __restrict__ dq, const float* __restrict__ gdq,
                                    const float* __restrict__ gpos, const float* __restrict__ gaxis,
                                    float* __restrict__ gdof) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * sk.D) return;
    const int b = i / sk.D, d = i % sk.D;
    float acc = 0.f;
    for (int e = sk.dof_off[d]; e < sk.dof_off[d + 1]; ++e) {
        const int j = sk.dof_joint[e];
        const float3 ax = ld3(gaxis + ((long long)b * sk.J + j) * 3);
        const float3 c = ld3(gpos + ((long long)b * sk.J + j) * 3);
        float gj = 0.f;
        for (int s = 0; s < sk.S; ++s) {
            if (!sk.in_chain[s * sk.J + j]) continue;
            const float* q = dq + ((long long)b * sk.S + s) * 8;
            const float4 r = f4(q), tq = f4(q + 4);
            const float3 t = dq_trans(r, tq);
            float4 dr, dt3;
            float3 dtv;
            if (sk.type[j] == kRevolute) {
                dr = mul4(qmul(make_float4(ax.x, ax.y, ax.z, 0.f), r), 0.5f);
                dtv = cross(ax, t - c);
            } else {
                dr = make_float4(0.f, 0.f, 0.f, 0.f);
                dtv = ax;
            }
            dt3 = add4(mul4(qmul(make_float4(dtv.x, dtv.y, dtv.z, 0.f), r), 0.5f),
                       mul4(qmul(make_float4(t.x, t.y, t.z, 0.f), dr), 0.5f));
            const float* g = gdq + ((long long)b * sk.S + s) * 8;
            gj += dot4(f4(g), dr) + dot4(f4(g + 4), dt3);
        }
        acc += sk.dof_w[e] * gj;
    }
    gdof[i] = acc;
}

}  // namespace
}  // namespace hc

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace hc;

struct hc_skin_s {
    int J = 0, D = 0, S = 0, K = 0, N = 0, E = 0;
    int parity = 1;
    DevBuf parent, type, offset, axis, jscale, dof_off, dof_joint, dof_w, skin_joint, skin_scale, t0inv, in_chain,
        skin_idx, base_v, base_n, base_v4, base_n4;
    DevBuf joints, params, skin_xf, mom, lbs_xf, gpos, gaxis, dq_ws, gdq;
    Skel skel() const {
        Skel s;
        s.J = J;
        s.D = D;
        s.S = S;
        s.K = K;
        s.N = N;
        s.parent = parent.as<int>();
        s.type = type.as<int>();
        s.offset = offset.as<float>();
        s.axis = axis.as<float>();
        s.jscale = jscale.as<float>();
        s.dof_off = dof_off.as<int>();
        s.dof_joint = dof_joint.as<int>();
        s.dof_w = dof_w.as<float>();
        s.skin_joint = skin_joint.as<int>();
        s.skin_scale = skin_scale.as<float>();
        s.t0inv = t0inv.as<float>();
        s.in_chain = in_chain.as<unsigned char>();
        s.skin_idx = skin_idx.as<int>();
        s.base_v = base_v.as<float>();
        s.base_n = base_n.as<float>();
        s.base_v4 = base_v4.as<float4>();
        s.base_n4 = base_n4.as<float4>();
        return s;
    }
};

// Opt a kernel in to more than 48 KB of dynamic shared memory, once per device.
template <typename K>
static hc_status skin_allow_smem(K kernel, size_t bytes) {
    static unsigned long long done = 0;  // one bit per device
    if (bytes <= (48u << 10)) return HC_OK;
    int dev = 0;
    HC_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && (done >> dev & 1ull)) return HC_OK;
    HC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    if (dev < 64) done |= 1ull << dev;
    return HC_OK;
}

// the skinning slots can be staged as int4 / float4: K a multiple of 4, 16-byte aligned arrays
static int slots_by_four(const hc_skin_s* h, const float* weights) {
    return h->K % 4 == 0 && ((uintptr_t)weights & 15) == 0 && ((uintptr_t)h->skin_idx.ptr & 15) == 0;
}

extern "C" hc_status hc_skin_create(hc_skin* out, int32_t n_joints, const int32_t* parent, const int32_t* joint_type,
                                    const float* offset, const float* axis, const float* joint_scale, int32_t n_dofs,
                                    const int32_t* dof_offsets, const int32_t* dof_joint, const float* dof_weight,
                                    int32_t n_skin, const int32_t* skin_joint, const float* skin_scale,
                                    int32_t n_vertices, const float* base_vertices, const float* base_normals,
                                    int32_t k, const int32_t* skin_index) {
    clear_error();
    HC_REQUIRE(out, "out is NULL");
    *out = nullptr;
    HC_REQUIRE(n_joints > 0 && n_dofs > 0 && n_skin > 0 && n_vertices > 0 && k > 0, "empty skeleton or mesh");
    HC_REQUIRE(n_skin <= 1024, "at most 1024 skinning joints (got %d)", n_skin);
    HC_REQUIRE(skin_block_smem(n_skin, 12, k, kSkinBlock) <= (200u << 10),
               "%d skinning joints with %d per vertex exceed the staged skinning block", n_skin, k);
    HC_REQUIRE(parent && joint_type && offset && axis && dof_offsets && dof_joint && dof_weight && skin_joint &&
                   base_vertices && base_normals && skin_index,
               "NULL skeleton / mesh array");
    for (int j = 0; j < n_joints; ++j) {
        HC_REQUIRE(parent[j] < j && parent[j] >= -1, "joint %d: parent %d must precede it", j, parent[j]);
        HC_REQUIRE(joint_type[j] == kRevolute || joint_type[j] == kPrismatic,
                   "joint %d: only revolute (0) and prismatic (1) joints are supported", j);
    }
    HC_REQUIRE(dof_offsets[0] == 0, "dof_offsets[0] must be 0");
    for (int d = 0; d < n_dofs; ++d) HC_REQUIRE(dof_offsets[d + 1] >= dof_offsets[d], "dof_offsets not monotone");
    const int E = dof_offsets[n_dofs];
    for (int e = 0; e < E; ++e) HC_REQUIRE(dof_joint[e] >= 0 && dof_joint[e] < n_joints, "dof joint out of range");
    for (int s = 0; s < n_skin; ++s)
        HC_REQUIRE(skin_joint[s] >= 0 && skin_joint[s] < n_joints, "skinning joint %d out of range", s);
    for (long long i = 0; i < (long long)n_vertices * k; ++i)
        HC_REQUIRE(skin_index[i] >= 0 && skin_index[i] < n_skin, "skin index out of range");
    std::vector<float> js(n_joints, 1.f), ss(n_skin, 1.f);
    if (joint_scale) js.assign(joint_scale, joint_scale + n_joints);
    if (skin_scale) ss.assign(skin_scale, skin_scale + n_skin);
    // inverse bind transforms of the skinning joints, the character's initial
    // transformations (skinnedcharacter.cpp:130-138, 178-183): the bind pose has
    // zero dofs and every joint scale set to 1 (skeleton.cpp:2840-2853); the
    // joint scales come back afterwards (skeleton.cpp:2857-2862)
    std::vector<double> TR(9 * (size_t)n_joints), TT(3 * (size_t)n_joints);
    for (int j = 0; j < n_joints; ++j) {
        double lt[3];
        for (int c = 0; c < 3; ++c) lt[c] = (double)offset[3 * j + c];
        const int p = parent[j];
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) TR[9 * j + 3 * r + c] = p >= 0 ? TR[9 * p + 3 * r + c] : (r == c);
            TT[3 * j + r] = p >= 0 ? TR[9 * p + 3 * r] * lt[0] + TR[9 * p + 3 * r + 1] * lt[1] +
                                         TR[9 * p + 3 * r + 2] * lt[2] + TT[3 * p + r]
                                   : lt[r];
        }
    }
    std::vector<float> t0(12 * (size_t)n_skin);
    std::vector<unsigned char> chain((size_t)n_skin * n_joints, 0);
    for (int s = 0; s < n_skin; ++s) {
        const int j = skin_joint[s];
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) t0[12 * s + 3 * r + c] = (float)TR[9 * j + 3 * c + r];  // R^T
            double acc = 0;
            for (int c = 0; c < 3; ++c) acc += TR[9 * j + 3 * c + r] * TT[3 * j + c];
            t0[12 * s + 9 + r] = (float)-acc;
        }
        for (int q = j; q >= 0; q = parent[q]) chain[(size_t)s * n_joints + q] = 1;
    }
    hc_skin_s* h = new hc_skin_s();
    h->J = n_joints;
    h->D = n_dofs;
    h->E = E;
    h->S = n_skin;
    h->K = k;
    h->N = n_vertices;
    hc_status st = HC_OK;
#define UP(buf, ptr, n) \
    if (st == HC_OK) st = upload(h->buf, ptr, (size_t)(n));
    UP(parent, parent, n_joints);
    UP(type, joint_type, n_joints);
    UP(offset, offset, 3LL * n_joints);
    UP(axis, axis, 3LL * n_joints);
    UP(jscale, js.data(), n_joints);
    UP(dof_off, dof_offsets, n_dofs + 1LL);
    UP(dof_joint, dof_joint, std::max(E, 1));
    UP(dof_w, dof_weight, std::max(E, 1));
    UP(skin_joint, skin_joint, n_skin);
    UP(skin_scale, ss.data(), n_skin);
    UP(t0inv, t0.data(), t0.size());
    UP(in_chain, chain.data(), chain.size());
    UP(skin_idx, skin_index, (long long)n_vertices * k);
    UP(base_v, base_vertices, 3LL * n_vertices);
    UP(base_n, base_normals, 3LL * n_vertices);
    {
        std::vector<float4> bv4((size_t)n_vertices), bn4((size_t)n_vertices);
        for (int v = 0; v < n_vertices; ++v) {
            bv4[v] = make_float4(base_vertices[3 * v], base_vertices[3 * v + 1], base_vertices[3 * v + 2], 0.f);
            bn4[v] = make_float4(base_normals[3 * v], base_normals[3 * v + 1], base_normals[3 * v + 2], 0.f);
        }
        UP(base_v4, bv4.data(), bv4.size());
        UP(base_n4, bn4.data(), bn4.size());
    }
#undef UP
    if (st != HC_OK) {
        delete h;
        return st;
    }
    *out = h;
    return HC_OK;
}

extern "C" hc_status hc_skin_destroy(hc_skin h) {
    clear_error();
    if (!h) return HC_OK;
    DevBuf* bufs[] = {&h->parent, &h->type, &h->offset, &h->axis, &h->jscale, &h->dof_off, &h->dof_joint, &h->dof_w,
                      &h->skin_joint, &h->skin_scale, &h->t0inv, &h->in_chain, &h->skin_idx, &h->base_v,
                      &h->base_n, &h->joints, &h->params, &h->skin_xf, &h->mom, &h->lbs_xf, &h->gpos, &h->gaxis,
                      &h->dq_ws, &h->gdq};
    for (DevBuf* b : bufs) b->release();
    delete h;
    return HC_OK;
}

extern "C" hc_status hc_skin_set_parity(hc_skin h, int32_t parity) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    h->parity = parity ? 1 : 0;
    return HC_OK;
}

static hc_status fk(hc_skin h, cudaStream_t s, int B, const float* dofs, float* gpos, float* gaxis) {
    HC_TRY(h->joints.ensure(sizeof(Xf) * (size_t)B * h->J));
    HC_TRY(h->params.ensure(sizeof(float) * (size_t)B * h->J));
    HC_TRY(h->skin_xf.ensure(sizeof(Xf) * (size_t)B * h->S));
    const size_t smem = sizeof(float) * (2 * (size_t)((h->J + 3) & ~3) + 2 * (size_t)((h->E + 3) & ~3)) +
                        2 * sizeof(Xf) * (size_t)h->J;
    HC_REQUIRE(smem <= 48 * 1024, "skeleton too large for the kinematics kernel (%d joints)", h->J);
    k_fk<<<B, 128, smem, s>>>(h->skel(), B, dofs, h->joints.as<Xf>(), gpos, gaxis, h->skin_xf.as<Xf>(),
                              h->params.as<float>());
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_skin_reserve(hc_skin h, int32_t batch) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "invalid handle or batch");
    HC_TRY(h->joints.ensure(sizeof(Xf) * (size_t)batch * h->J));
    HC_TRY(h->params.ensure(sizeof(float) * (size_t)batch * h->J));
    HC_TRY(h->skin_xf.ensure(sizeof(Xf) * (size_t)batch * h->S));
    HC_TRY(h->mom.ensure(sizeof(float) * 6 * (size_t)batch * h->S));
    HC_TRY(h->lbs_xf.ensure(sizeof(float) * 12 * (size_t)batch * h->S));
    HC_TRY(h->gpos.ensure(sizeof(float) * 3 * (size_t)batch * h->J));
    HC_TRY(h->gaxis.ensure(sizeof(float) * 3 * (size_t)batch * h->J));
    return HC_OK;
}

extern "C" hc_status hc_dq_skinning_forward(hc_skin h, void* stream, int32_t batch, const float* dofs,
                                            const float* skinning_weights, float* skinned_vertex_positions,
                                            float* skinned_vertex_normals, float* global_joint_position,
                                            float* global_joint_axis, float* dual_quaternions,
                                            float* output_skinning_weights) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "invalid handle or batch");
    HC_REQUIRE(dofs && skinning_weights && skinned_vertex_positions && skinned_vertex_normals &&
                   global_joint_position && global_joint_axis && dual_quaternions,
               "NULL input/output pointer");
    cudaStream_t s = (cudaStream_t)stream;
    HC_TRY(fk(h, s, batch, dofs, global_joint_position, global_joint_axis));
    const int BS = batch * h->S;
    k_dq_from_xf<<<div_up(BS, 128), 128, 0, s>>>(BS, h->skin_xf.as<Xf>(), dual_quaternions);
    HC_CHECK_LAUNCH();
    HC_REQUIRE(batch <= 65535, "too many frames in one call (%d)", batch);
    HC_TRY(skin_allow_smem(k_dq_skin, skin_block_smem(h->S, 8, h->K, kSkinBlock)));
    k_dq_skin<<<dim3(div_up(h->N, kSkinBlock), batch), kSkinBlock, skin_block_smem(h->S, 8, h->K, kSkinBlock), s>>>(
        h->skel(), batch, dual_quaternions, skinning_weights, skinned_vertex_positions, skinned_vertex_normals,
        output_skinning_weights, slots_by_four(h, skinning_weights));
    HC_CHECK_LAUNCH();
    return HC_OK;
}

static hc_status dof_grad(hc_skin h, cudaStream_t s, int B, const float* vpos, const float* gv, const float* w,
                          const float* gpos, const float* gaxis, float* gdof) {
    HC_TRY(h->mom.ensure(sizeof(float) * 6 * (size_t)B * h->S));
    HC_CUDA(cudaMemsetAsync(h->mom.ptr, 0, sizeof(float) * 6 * (size_t)B * h->S, s));
    const dim3 grid(div_up(h->N, 256), B);
    k_bone_moments<<<grid, 256, sizeof(float) * 6 * h->S, s>>>(h->skel(), vpos, gv, w, h->mom.as<float>());
    HC_CHECK_LAUNCH();
    k_dof_grad<<<div_up(B * h->D, 128), 128, 0, s>>>(h->skel(), B, h->mom.as<float>(), gpos, gaxis, gdof);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_dq_skinning_backward(hc_skin h, void* stream, int32_t batch,
                                             const float* skinned_vertex_positions_grad,
                                             const float* skinned_vertex_positions, const float* global_joint_position,
                                             const float* global_joint_axis, const float* dual_quaternions,
                                             const float* skinning_weights, float* dofs_grad,
                                             float* skinning_weights_grad) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "invalid handle or batch");
    HC_REQUIRE(skinned_vertex_positions_grad && skinned_vertex_positions && global_joint_position &&
                   global_joint_axis && dual_quaternions && skinning_weights && dofs_grad && skinning_weights_grad,
               "NULL input/output pointer");
    cudaStream_t s = (cudaStream_t)stream;
    HC_TRY(dof_grad(h, s, batch, skinned_vertex_positions, skinned_vertex_positions_grad, skinning_weights,
                    global_joint_position, global_joint_axis, dofs_grad));
    const long long n = (long long)batch * h->N * h->K;
    k_dq_weight_grad<<<div_up(n, 128), 128, 0, s>>>(h->skel(), batch, dual_quaternions, skinning_weights,
                                                    skinned_vertex_positions_grad, h->parity, skinning_weights_grad);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_lb_skinning_forward(hc_skin h, void* stream, int32_t batch, const float* dofs,
                                            const float* skinning_weights, const float* displacement,
                                            float* skinned_vertex_positions, float* skinned_vertex_normals,
                                            float* global_joint_position, float* global_joint_axis,
                                            float* transformation, float* output_skinning_weights) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "invalid handle or batch");
    HC_REQUIRE(dofs && skinning_weights && displacement && skinned_vertex_positions && skinned_vertex_normals &&
                   global_joint_position && global_joint_axis && transformation,
               "NULL input/output pointer");
    cudaStream_t s = (cudaStream_t)stream;
    HC_TRY(fk(h, s, batch, dofs, global_joint_position, global_joint_axis));
    const int BS = batch * h->S;
    k_xf_to_lbs<<<div_up(BS, 128), 128, 0, s>>>(BS, h->skin_xf.as<Xf>(), transformation);
    HC_CHECK_LAUNCH();
    HC_REQUIRE(batch <= 65535, "too many frames in one call (%d)", batch);
    HC_TRY(skin_allow_smem(k_lbs_skin, skin_block_smem(h->S, 12, h->K, kSkinBlock)));
    k_lbs_skin<<<dim3(div_up(h->N, kSkinBlock), batch), kSkinBlock, skin_block_smem(h->S, 12, h->K, kSkinBlock), s>>>(
        h->skel(), batch, transformation, skinning_weights, displacement, skinned_vertex_positions,
        skinned_vertex_normals, output_skinning_weights, slots_by_four(h, skinning_weights));
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_lb_skinning_backward(hc_skin h, void* stream, int32_t batch,
                                             const float* skinned_vertex_positions_grad,
                                             const float* skinned_vertex_positions, const float* global_joint_position,
                                             const float* global_joint_axis, const float* transformation,
                                             const float* skinning_weights, const float* displacement,
                                             float* dofs_grad, float* skinning_weights_grad,
                                             float* displacement_grad) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "invalid handle or batch");
    HC_REQUIRE(skinned_vertex_positions_grad && skinned_vertex_positions && global_joint_position &&
                   global_joint_axis && transformation && skinning_weights && dofs_grad && skinning_weights_grad &&
                   displacement_grad,
               "NULL input/output pointer");
    HC_REQUIRE(h->parity || displacement, "the exact LBS weight gradient needs the displacement input");
    cudaStream_t s = (cudaStream_t)stream;
    HC_TRY(dof_grad(h, s, batch, skinned_vertex_positions, skinned_vertex_positions_grad, skinning_weights,
                    global_joint_position, global_joint_axis, dofs_grad));
    const long long n = (long long)batch * h->N * h->K;
    k_lbs_weight_grad<<<div_up(n, 128), 128, 0, s>>>(h->skel(), batch, transformation, displacement,
                                                     skinned_vertex_positions_grad, h->parity, skinning_weights_grad);
    HC_CHECK_LAUNCH();
    k_lbs_disp_grad<<<div_up((long long)batch * h->N, 128), 128, 0, s>>>(
        h->skel(), batch, transformation, skinning_weights, skinned_vertex_positions_grad, h->parity,
        displacement_grad);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_pose2eg_forward(hc_skin h, void* stream, int32_t batch, const float* dofs, int32_t n_nodes,
                                        const int32_t* node_vertex, const float* vertex_weights,
                                        float* nodes_skinned_translation, float* nodes_skinned_rotation,
                                        float* dual_quaternions) {
    clear_error();
    HC_REQUIRE(h && batch > 0 && n_nodes > 0, "invalid handle or sizes");
    HC_REQUIRE(dofs && node_vertex && vertex_weights && nodes_skinned_translation && nodes_skinned_rotation &&
                   dual_quaternions,
               "NULL pointer");
    cudaStream_t s = (cudaStream_t)stream;
    HC_TRY(h->gpos.ensure(sizeof(float) * 3 * (size_t)batch * h->J));
    HC_TRY(h->gaxis.ensure(sizeof(float) * 3 * (size_t)batch * h->J));
    HC_TRY(fk(h, s, batch, dofs, h->gpos.as<float>(), h->gaxis.as<float>()));
    const int BS = batch * h->S;
    k_dq_from_xf<<<div_up(BS, 128), 128, 0, s>>>(BS, h->skin_xf.as<Xf>(), dual_quaternions);
    HC_CHECK_LAUNCH();
    k_pose2eg<<<div_up((long long)batch * n_nodes, 128), 128, 0, s>>>(h->skel(), batch, n_nodes, node_vertex,
                                                                       dual_quaternions, vertex_weights,
                                                                       nodes_skinned_translation,
                                                                       nodes_skinned_rotation);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_pose2eg_backward(hc_skin h, void* stream, int32_t batch, const float* dofs, int32_t n_nodes,
                                         const int32_t* node_vertex, const float* vertex_weights,
                                         const float* nodes_skinned_translation_grad,
                                         const float* nodes_skinned_rotation_grad, float* dofs_grad) {
    clear_error();
    HC_REQUIRE(h && batch > 0 && n_nodes > 0, "invalid handle or sizes");
    HC_REQUIRE(dofs && node_vertex && vertex_weights && nodes_skinned_translation_grad &&
                   nodes_skinned_rotation_grad && dofs_grad,
               "NULL pointer");
    HC_REQUIRE(h->K <= 16, "node skinning gradient supports up to 16 skinning joints per vertex");
    HC_REQUIRE(batch <= 65535, "batch %d above 65535", batch);
    cudaStream_t s = (cudaStream_t)stream;
    HC_TRY(hc_skin_reserve(h, batch));
    HC_TRY(h->dq_ws.ensure(sizeof(float) * 8 * (size_t)batch * h->S));
    HC_TRY(h->gdq.ensure(sizeof(float) * 8 * (size_t)batch * h->S));
    HC_TRY(fk(h, s, batch, dofs, h->gpos.as<float>(), h->gaxis.as<float>()));
    const int BS = batch * h->S;
    k_dq_from_xf<<<div_up(BS, 128), 128, 0, s>>>(BS, h->skin_xf.as<Xf>(), h->dq_ws.as<float>());
    HC_CHECK_LAUNCH();
    const size_t smem = sizeof(float) * 8 * (size_t)h->S * 4;  // 4 warps
    HC_REQUIRE(smem <= 48 * 1024, "too many skinning joints (%d)", h->S);
    HC_CUDA(cudaMemsetAsync(h->gdq.ptr, 0, sizeof(float) * 8 * (size_t)batch * h->S, s));
    const dim3 grid((unsigned)std::min(div_up(n_nodes, 128), 64), (unsigned)batch);
    k_pose2eg_grad_nodes<<<grid, 128, smem, s>>>(h->skel(), n_nodes, node_vertex, h->dq_ws.as<float>(),
                                                  vertex_weights, nodes_skinned_translation_grad,
                                                  nodes_skinned_rotation_grad, h->gdq.as<float>());
    HC_CHECK_LAUNCH();
    k_pose2eg_grad_dofs<<<div_up(batch * h->D, 128), 128, 0, s>>>(h->skel(), batch, h->dq_ws.as<float>(),
                                                                  h->gdq.as<float>(), h->gpos.as<float>(),
                                                                  h->gaxis.as<float>(), dofs_grad);
    HC_CHECK_LAUNCH();
    return HC_OK;
}
