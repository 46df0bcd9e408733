// Image loss of the training step: masked L1 on 255-scaled colours, divided
// by the number of non-zero residual entries (Projects/HoloportedCharacters/
// HPCMeshDL.py:669-688: difference = 255 (R - T) * mask * model_mask,
// loss = sum |difference| / count_nonzero(difference)), and its gradient
// d loss / d R = 255 sign(difference) * mask * model_mask / count
// (the count is a constant for the gradient, as in TF).
#include <algorithm>
#include <math.h>

#include "hc_common.cuh"
#include "hc_math.cuh"

namespace hc {
namespace {

using L1Acc = L1State;

__global__ void k_l1_reduce(long long n_px, const float* __restrict__ render, const float* __restrict__ target,
                            const int* __restrict__ face, const unsigned char* __restrict__ mask,
                            L1Acc* __restrict__ acc) {
    float s = 0.f;
    unsigned cnt = 0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n_px;
         p += (long long)gridDim.x * blockDim.x) {
        const bool m = face[p] >= 0 && (!mask || mask[p]);
        if (!m) continue;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float d = l1_diff(render[3 * p + c], target[3 * p + c]);
            s += fabsf(d);
            cnt += d != 0.f;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    __shared__ float ss[32];
    __shared__ unsigned sc[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        ss[w] = s;
        sc[w] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        unsigned long long c = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            t += ss[i];
            c += sc[i];
        }
        atomicAdd(&acc->sum, t);
        atomicAdd(&acc->count, c);
    }
}

__global__ void k_l1_grad(long long n_px, const float* __restrict__ render, const float* __restrict__ target,
                          const int* __restrict__ face, const unsigned char* __restrict__ mask,
                          const L1Acc* __restrict__ acc, float* __restrict__ grad, float* __restrict__ loss) {
    const unsigned long long cnt = acc->count;
    const float scale = cnt ? 255.f / (float)cnt : 0.f;
    if (blockIdx.x == 0 && threadIdx.x == 0 && loss) *loss = cnt ? (float)(acc->sum / (double)cnt) : 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n_px;
         p += (long long)gridDim.x * blockDim.x) {
        const bool m = face[p] >= 0 && (!mask || mask[p]);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float g = 0.f;
            if (m) {
                g = l1_grad(l1_diff(render[3 * p + c], target[3 * p + c]), scale);
            }
            grad[3 * p + c] = g;
        }
    }
}

// one pass: grad = 2 w x and the block partials of sum x^2 (vec: 16-byte
// loads and stores, n a multiple of 4 and both pointers 16-byte aligned)
__global__ void k_sumsq_fused(long long n, const float* __restrict__ x, float weight, double* __restrict__ acc,
                              float* __restrict__ grad, int vec) {
    const float k = 2.f * weight;
    float s = 0.f;
    const long long stride = (long long)gridDim.x * blockDim.x;
    if (vec) {
        const float4* x4 = reinterpret_cast<const float4*>(x);
        float4* g4 = reinterpret_cast<float4*>(grad);
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n / 4; i += stride) {
            const float4 v = x4[i];
            s += v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w;
            g4[i] = make_float4(k * v.x, k * v.y, k * v.z, k * v.w);
        }
    } else {
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
            const float v = x[i];
            s += v * v;
            grad[i] = k * v;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float ss[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ss[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += ss[i];
        atomicAdd(acc, t);
    }
}

__global__ void k_sumsq_loss(float weight, const double* __restrict__ acc, float* __restrict__ loss) {
    *loss = (float)(weight * *acc);
}

__global__ void k_add_inplace(long long n, float* __restrict__ dst, const float* __restrict__ src) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] += src[i];
}

// 8-bit image values -> float32 in [0, 1] (k / 255, IEEE division); four
// bytes per thread and step
__global__ void k_u8_to_f32(long long n, const unsigned char* __restrict__ src, float* __restrict__ dst) {
    const long long n4 = n / 4;
    const uchar4* s4 = reinterpret_cast<const uchar4*>(src);
    float4* d4 = reinterpret_cast<float4*>(dst);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
        const uchar4 q = s4[i];
        d4[i] = make_float4((float)q.x / 255.f, (float)q.y / 255.f, (float)q.z / 255.f, (float)q.w / 255.f);
    }
    for (long long i = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = (float)src[i] / 255.f;
}

// Gaussian smoothing of images (Projects/CustomTFOperators/GaussianSmoothingGpu.py:12-37):
// a depthwise (2s+1)^2 convolution with the normalised outer product of a
// sampled normal density, zero padding ("SAME").  The kernel is separable, so
// each CTA stages a 32x32 output tile with its halo in shared memory and runs
// a horizontal then a vertical pass: one read and one write of the image.
constexpr int kSmoothTile = 32;
constexpr int kSmoothMax = 15;

struct SmoothTaps {
    float w[2 * kSmoothMax + 1];
};

__global__ void k_smooth(int H, int W, int Cn, int s, SmoothTaps taps, const float* __restrict__ in,
                         float* __restrict__ out) {
    extern __shared__ float sm[];
    const int E = kSmoothTile + 2 * s;
    float* s_in = sm;                       // [E][E][Cn]
    float* s_h = sm + (size_t)E * E * Cn;   // [E][32][Cn]
    const int img = blockIdx.z;
    const int x0 = blockIdx.x * kSmoothTile - s, y0 = blockIdx.y * kSmoothTile - s;
    const float* I = in + (long long)img * H * W * Cn;
    for (int i = threadIdx.x; i < E * E * Cn; i += blockDim.x) {
        const int c = i % Cn, p = i / Cn, xx = x0 + p % E, yy = y0 + p / E;
        s_in[i] = (xx >= 0 && yy >= 0 && xx < W && yy < H) ? I[((long long)yy * W + xx) * Cn + c] : 0.f;
    }
    __syncthreads();
    const int n = 2 * s + 1;
    for (int i = threadIdx.x; i < E * kSmoothTile * Cn; i += blockDim.x) {
        const int c = i % Cn, p = i / Cn, x = p % kSmoothTile, y = p / kSmoothTile;
        const float* row = s_in + ((size_t)y * E + x) * Cn + c;
        float acc = 0.f;
        for (int k = 0; k < n; ++k) acc += taps.w[k] * row[k * Cn];
        s_h[i] = acc;
    }
    __syncthreads();
    float* O = out + (long long)img * H * W * Cn;
    for (int i = threadIdx.x; i < kSmoothTile * kSmoothTile * Cn; i += blockDim.x) {
        const int c = i % Cn, p = i / Cn, x = p % kSmoothTile, y = p / kSmoothTile;
        const int gx = blockIdx.x * kSmoothTile + x, gy = blockIdx.y * kSmoothTile + y;
        if (gx >= W || gy >= H) continue;
        const float* col = s_h + ((size_t)y * kSmoothTile + x) * Cn + c;
        float acc = 0.f;
        for (int k = 0; k < n; ++k) acc += taps.w[k] * col[(size_t)k * kSmoothTile * Cn];
        O[((long long)gy * W + gx) * Cn + c] = acc;
    }
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_gaussian_smooth(void* stream, int32_t n_images, int32_t height, int32_t width,
                                        int32_t channels, int32_t size, float mean, float std, const float* image,
                                        float* out) {
    clear_error();
    HC_REQUIRE(n_images >= 0 && height > 0 && width > 0 && channels > 0 && channels <= 4, "bad sizes");
    HC_REQUIRE(size >= 0 && size <= kSmoothMax, "kernel size %d outside [0, %d]", size, kSmoothMax);
    HC_REQUIRE(image && out, "NULL pointer");
    HC_REQUIRE(image != out || size == 0 || std == 0.f, "in-place smoothing is not supported");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = sizeof(float) * (size_t)n_images * height * width * channels;
    if (size == 0 || std == 0.f) {  // the reference returns the image unchanged
        if (image != out && bytes) HC_CUDA(cudaMemcpyAsync(out, image, bytes, cudaMemcpyDeviceToDevice, s));
        return HC_OK;
    }
    if (n_images == 0) return HC_OK;
    // normal density at -size..size, normalised so the 2-D kernel sums to one
    SmoothTaps t;
    double v[2 * kSmoothMax + 1], sum = 0.0;
    for (int k = 0; k <= 2 * size; ++k) {
        const double z = ((double)(k - size) - mean) / std;
        v[k] = exp(-0.5 * z * z);
        sum += v[k];
    }
    for (int k = 0; k <= 2 * size; ++k) t.w[k] = (float)(v[k] / sum);
    const int E = kSmoothTile + 2 * size;
    const size_t smem = sizeof(float) * ((size_t)E * E + (size_t)E * kSmoothTile) * channels;
    HC_CUDA(cudaFuncSetAttribute(k_smooth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 grid(div_up(width, kSmoothTile), div_up(height, kSmoothTile), n_images);
    k_smooth<<<grid, 256, smem, s>>>(height, width, channels, size, t, image, out);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_sum_squares_loss(void* stream, int64_t n, const float* x, float weight, void* workspace,
                                         float* loss, float* grad) {
    clear_error();
    HC_REQUIRE(n >= 0, "n < 0");
    HC_REQUIRE(x && workspace && grad, "NULL input/output pointer");
    cudaStream_t s = (cudaStream_t)stream;
    double* acc = (double*)workspace;
    HC_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), s));
    // grid-stride: as many CTAs as are resident at once, so that no partial
    // second wave runs after the rest
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sumsq_fused, 256, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    const int blocks = (int)std::max<long long>(1, std::min<long long>((long long)sms * per_sm, n / 1024 + 1));
    const int vec = n % 4 == 0 && ((uintptr_t)x & 15) == 0 && ((uintptr_t)grad & 15) == 0;
    k_sumsq_fused<<<blocks, 256, 0, s>>>(n, x, weight, acc, grad, vec);
    HC_CHECK_LAUNCH();
    if (loss) {
        k_sumsq_loss<<<1, 1, 0, s>>>(weight, acc, loss);
        HC_CHECK_LAUNCH();
    }
    return HC_OK;
}

extern "C" hc_status hc_add_inplace(void* stream, int64_t n, float* dst, const float* src) {
    clear_error();
    HC_REQUIRE(n >= 0, "n < 0");
    HC_REQUIRE(dst && src, "NULL pointer");
    if (n == 0) return HC_OK;
    const long long blocks = n / 1024 + 1 < 148 * 8 ? n / 1024 + 1 : 148 * 8;
    k_add_inplace<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(n, dst, src);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_image_u8_to_f32(void* stream, int64_t n, const uint8_t* src, float* dst) {
    clear_error();
    HC_REQUIRE(n >= 0, "n < 0");
    HC_REQUIRE(src && dst, "NULL pointer");
    HC_REQUIRE(((uintptr_t)src & 3) == 0 && ((uintptr_t)dst & 15) == 0,
               "src must be 4-byte and dst 16-byte aligned");
    if (n == 0) return HC_OK;
    const long long blocks = n / 4096 + 1 < 148 * 8 ? n / 4096 + 1 : 148 * 8;
    k_u8_to_f32<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(n, src, dst);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_image_l1_loss(void* stream, int64_t n_pixels, const float* render_buffer,
                                      const float* target_image, const int32_t* face_buffer,
                                      const uint8_t* foreground_mask, void* workspace, float* loss,
                                      float* render_buffer_grad) {
    clear_error();
    HC_REQUIRE(n_pixels >= 0, "n_pixels < 0");
    HC_REQUIRE(render_buffer && target_image && face_buffer && workspace && render_buffer_grad,
               "NULL input/output pointer");
    cudaStream_t s = (cudaStream_t)stream;
    L1Acc* acc = (L1Acc*)workspace;
    HC_CUDA(cudaMemsetAsync(acc, 0, sizeof(L1Acc), s));
    const int blocks = 148 * 8;
    k_l1_reduce<<<blocks, 256, 0, s>>>(n_pixels, render_buffer, target_image, face_buffer, foreground_mask, acc);
    HC_CHECK_LAUNCH();
    k_l1_grad<<<blocks, 256, 0, s>>>(n_pixels, render_buffer, target_image, face_buffer, foreground_mask, acc,
                                     render_buffer_grad, loss);
    HC_CHECK_LAUNCH();
    return HC_OK;
}
