// Image loss of the training step: masked L1 on 255-scaled colours, divided
// by the number of non-zero residual entries (Projects/HoloportedCharacters/
// HPCMeshDL.py:669-688: difference = 255 (R - T) * mask * model_mask,
// loss = sum |difference| / count_nonzero(difference)), and its gradient
// d loss / d R = 255 sign(difference) * mask * model_mask / count
// (the count is a constant for the gradient, as in TF).
#include "hc_common.cuh"

namespace hc {
namespace {

struct L1Acc {
    double sum;
    unsigned long long count;
};

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
            const float d = 255.f * render[3 * p + c] - 255.f * target[3 * p + c];
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
                const float d = 255.f * render[3 * p + c] - 255.f * target[3 * p + c];
                g = d > 0.f ? scale : (d < 0.f ? -scale : 0.f);
            }
            grad[3 * p + c] = g;
        }
    }
}

}  // namespace
}  // namespace hc

using namespace hc;

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
