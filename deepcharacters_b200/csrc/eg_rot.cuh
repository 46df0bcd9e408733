// Euler rotations of the embedded graph, shared by the deformation and the
// ARAP regulariser: R(a) = Rz(a.z) Ry(a.y) Rx(a.x) and its partial
// derivatives (CustomTensorFlowCPPOperators/src/CudaUtils/
// EmbeddedGraphRotationHelper.h:53-191), with the reference's operation order.
#pragma once
#include <cuda_runtime.h>

namespace hc {

struct R33 {
    float m[9];  // row-major
};

// R = Rz(c) Ry(b) Rx(a) (EmbeddedGraphRotationHelper.h:53-77)
__device__ __forceinline__ R33 euler_rot(float3 a) {
    const float ca = cos(a.x), cb = cos(a.y), cg = cos(a.z);
    const float sa = sin(a.x), sb = sin(a.y), sg = sin(a.z);
    R33 R;
    R.m[0] = cb * cg;
    R.m[1] = sa * sb * cg - ca * sg;
    R.m[2] = ca * sb * cg + sa * sg;
    R.m[3] = cb * sg;
    R.m[4] = sa * sb * sg + ca * cg;
    R.m[5] = ca * sb * sg - sa * cg;
    R.m[6] = -sb;
    R.m[7] = sa * cb;
    R.m[8] = ca * cb;
    return R;
}

// dR/da, dR/db, dR/dc (EmbeddedGraphRotationHelper.h:109-191)
__device__ __forceinline__ void euler_rot_d(float3 a, R33& da, R33& db, R33& dc) {
    const float ca = cos(a.x), cb = cos(a.y), cg = cos(a.z);
    const float sa = sin(a.x), sb = sin(a.y), sg = sin(a.z);
    da.m[0] = 0.f;
    da.m[1] = ca * sb * cg + sa * sg;
    da.m[2] = -sa * sb * cg + ca * sg;
    da.m[3] = 0.f;
    da.m[4] = ca * sb * sg - sa * cg;
    da.m[5] = -sa * sb * sg - ca * cg;
    da.m[6] = 0.f;
    da.m[7] = ca * cb;
    da.m[8] = -sa * cb;
    db.m[0] = -sb * cg;
    db.m[1] = sa * cb * cg;
    db.m[2] = ca * cb * cg;
    db.m[3] = -sb * sg;
    db.m[4] = sa * cb * sg;
    db.m[5] = ca * cb * sg;
    db.m[6] = -cb;
    db.m[7] = -sa * sb;
    db.m[8] = -ca * sb;
    dc.m[0] = -cb * sg;
    dc.m[1] = -sa * sb * sg - ca * cg;
    dc.m[2] = -ca * sb * sg + sa * cg;
    dc.m[3] = cb * cg;
    dc.m[4] = sa * sb * cg - ca * sg;
    dc.m[5] = ca * sb * cg + sa * sg;
    dc.m[6] = 0.f;
    dc.m[7] = 0.f;
    dc.m[8] = 0.f;
}

__device__ __forceinline__ float3 mv(const R33& R, float3 v) {
    return make_float3(R.m[0] * v.x + R.m[1] * v.y + R.m[2] * v.z, R.m[3] * v.x + R.m[4] * v.y + R.m[5] * v.z,
                       R.m[6] * v.x + R.m[7] * v.y + R.m[8] * v.z);
}

}  // namespace hc
