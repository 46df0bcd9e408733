// Small vector / matrix helpers shared by the kernels.
//
// The rasterizer reproduces the reference's per-pixel float arithmetic so that
// visibility decisions agree bit for bit.  The helpers below therefore keep
// the plain left-to-right operation order of the reference's vector maths
// (dot = x*x' + y*y' + z*z', cross = (ay*bz - az*by, ...), normalize =
// v * rsqrtf(dot(v, v))), and this file must be compiled without fast-math so
// that divisions stay IEEE-rounded.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define HC_HD __host__ __device__ __forceinline__

HC_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
HC_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
HC_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
HC_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
HC_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
HC_HD float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
HC_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
HC_HD float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
HC_HD void operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
HC_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HC_HD float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
HC_HD float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
HC_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
HC_HD float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }


// Quotient and remainder of 32-bit unsigned integers by a divisor that is
// fixed for a launch, as a multiply-high and two shifts instead of the
// emulated integer division.  Method: Granlund and Montgomery, "Division by
// invariant integers using multiplication" (PLDI 1994), figure 4.1: for
// 1 <= d < 2^32 with l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// sh1 = min(l, 1), sh2 = max(l - 1, 0), every n < 2^32 has
// n / d = (t + ((n - t) >> sh1)) >> sh2 with t = mulhi(m, n).
struct FastDiv {
    unsigned d = 1, m = 1, sh1 = 0, sh2 = 0;
    FastDiv() = default;
    explicit FastDiv(unsigned divisor) : d(divisor ? divisor : 1u) {
        unsigned l = 0;
        while (l < 32 && (1ull << l) < d) ++l;
        m = (unsigned)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
        sh1 = l < 1 ? l : 1u;
        sh2 = l > 1 ? l - 1 : 0u;
    }
#ifdef __CUDACC__
    __device__ __forceinline__ unsigned div(unsigned n) const {
        const unsigned t = __umulhi(m, n);
        return (t + ((n - t) >> sh1)) >> sh2;
    }
    __device__ __forceinline__ unsigned mod(unsigned n, unsigned q) const { return n - q * d; }
#endif
};

#ifdef __CUDACC__
__device__ __forceinline__ float length3(float3 v) { return sqrtf(dot(v, v)); }
__device__ __forceinline__ float3 normalize3(float3 v) {
    float inv = rsqrtf(dot(v, v));
    return v * inv;
}
#endif

HC_HD float3 ld3(const float* p) { return make_float3(p[0], p[1], p[2]); }
HC_HD void st3(float* p, float3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

// Row-major 4x4 matrix.
struct M44 {
    float e[16];
};

// Product of two row-major 4x4 matrices, every entry as the full four-term
// sum r_ij = a_i0*b_0j + a_i1*b_1j + a_i2*b_2j + a_i3*b_3j (zeros included).
HC_HD M44 mul44(const M44& a, const M44& b) {
    M44 r;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
            r.e[4 * i + j] = a.e[4 * i + 0] * b.e[0 + j] + a.e[4 * i + 1] * b.e[4 + j] +
                             a.e[4 * i + 2] * b.e[8 + j] + a.e[4 * i + 3] * b.e[12 + j];
    return r;
}

// Inverse by the adjugate (cofactor expansion of each 3x3 minor, determinant
// along the first row, one reciprocal).  This is the textbook closed form
// also used by the reference camera set-up
// (CudaRenderer/cpp/src/Utils/float4x4.h:160-285); the cofactor sums keep
// that term order so that inverse camera matrices match bit for bit.
HC_HD M44 inverse44(const M44& m) {
    const float* x = m.e;
    float inv[16];
    inv[0] = x[5] * x[10] * x[15] - x[5] * x[11] * x[14] - x[9] * x[6] * x[15] +
             x[9] * x[7] * x[14] + x[13] * x[6] * x[11] - x[13] * x[7] * x[10];
    inv[4] = -x[4] * x[10] * x[15] + x[4] * x[11] * x[14] + x[8] * x[6] * x[15] -
             x[8] * x[7] * x[14] - x[12] * x[6] * x[11] + x[12] * x[7] * x[10];
    inv[8] = x[4] * x[9] * x[15] - x[4] * x[11] * x[13] - x[8] * x[5] * x[15] +
             x[8] * x[7] * x[13] + x[12] * x[5] * x[11] - x[12] * x[7] * x[9];
    inv[12] = -x[4] * x[9] * x[14] + x[4] * x[10] * x[13] + x[8] * x[5] * x[14] -
              x[8] * x[6] * x[13] - x[12] * x[5] * x[10] + x[12] * x[6] * x[9];
    inv[1] = -x[1] * x[10] * x[15] + x[1] * x[11] * x[14] + x[9] * x[2] * x[15] -
             x[9] * x[3] * x[14] - x[13] * x[2] * x[11] + x[13] * x[3] * x[10];
    inv[5] = x[0] * x[10] * x[15] - x[0] * x[11] * x[14] - x[8] * x[2] * x[15] +
             x[8] * x[3] * x[14] + x[12] * x[2] * x[11] - x[12] * x[3] * x[10];
    inv[9] = -x[0] * x[9] * x[15] + x[0] * x[11] * x[13] + x[8] * x[1] * x[15] -
             x[8] * x[3] * x[13] - x[12] * x[1] * x[11] + x[12] * x[3] * x[9];
    inv[13] = x[0] * x[9] * x[14] - x[0] * x[10] * x[13] - x[8] * x[1] * x[14] +
              x[8] * x[2] * x[13] + x[12] * x[1] * x[10] - x[12] * x[2] * x[9];
    inv[2] = x[1] * x[6] * x[15] - x[1] * x[7] * x[14] - x[5] * x[2] * x[15] +
             x[5] * x[3] * x[14] + x[13] * x[2] * x[7] - x[13] * x[3] * x[6];
    inv[6] = -x[0] * x[6] * x[15] + x[0] * x[7] * x[14] + x[4] * x[2] * x[15] -
             x[4] * x[3] * x[14] - x[12] * x[2] * x[7] + x[12] * x[3] * x[6];
    inv[10] = x[0] * x[5] * x[15] - x[0] * x[7] * x[13] - x[4] * x[1] * x[15] +
              x[4] * x[3] * x[13] + x[12] * x[1] * x[7] - x[12] * x[3] * x[5];
    inv[14] = -x[0] * x[5] * x[14] + x[0] * x[6] * x[13] + x[4] * x[1] * x[14] -
              x[4] * x[2] * x[13] - x[12] * x[1] * x[6] + x[12] * x[2] * x[5];
    inv[3] = -x[1] * x[6] * x[11] + x[1] * x[7] * x[10] + x[5] * x[2] * x[11] -
             x[5] * x[3] * x[10] - x[9] * x[2] * x[7] + x[9] * x[3] * x[6];
    inv[7] = x[0] * x[6] * x[11] - x[0] * x[7] * x[10] - x[4] * x[2] * x[11] +
             x[4] * x[3] * x[10] + x[8] * x[2] * x[7] - x[8] * x[3] * x[6];
    inv[11] = -x[0] * x[5] * x[11] + x[0] * x[7] * x[9] + x[4] * x[1] * x[11] -
              x[4] * x[3] * x[9] - x[8] * x[1] * x[7] + x[8] * x[3] * x[5];
    inv[15] = x[0] * x[5] * x[10] - x[0] * x[6] * x[9] - x[4] * x[1] * x[10] +
              x[4] * x[2] * x[9] + x[8] * x[1] * x[6] - x[8] * x[2] * x[5];
    float det = x[0] * inv[0] + x[1] * inv[4] + x[2] * inv[8] + x[3] * inv[12];
    float rdet = 1.0f / det;
    M44 r;
#pragma unroll
    for (int i = 0; i < 16; ++i) r.e[i] = inv[i] * rdet;
    return r;
}

// Masked image L1 of the training step (Projects/HoloportedCharacters/
// HPCMeshDL.py:642-688).  One channel's difference: render and target scaled
// by 255 and then subtracted, each product rounded on its own as the separate
// TF ops do (no fused multiply-add).
__device__ __forceinline__ float l1_diff(float r, float t) {
    return __fsub_rn(__fmul_rn(255.f, r), __fmul_rn(255.f, t));
}
// d loss / d render of one channel: 255 sign(difference) / count, scale = 255 / count
__device__ __forceinline__ float l1_grad(float d, float scale) { return d > 0.f ? scale : (d < 0.f ? -scale : 0.f); }

// Running L1 state (16 bytes, the workspace of the L1 entry points): the sum
// of |difference| and the number of non-zero differences.
struct L1State {
    double sum;
    unsigned long long count;
};
