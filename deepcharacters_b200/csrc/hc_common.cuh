// Runtime plumbing shared by the C-ABI entry points: status codes, the
// per-thread error message, CUDA error checks and a grow-only device buffer.
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "../../include/hc.h"

namespace hc {

void set_error(const char* fmt, ...);
void clear_error();
// process-wide count of kernel launches issued by this library
void count_launch();

#define HC_FAIL(code, ...)            \
    do {                              \
        ::hc::set_error(__VA_ARGS__); \
        return (code);                \
    } while (0)

#define HC_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            HC_FAIL(HC_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    } while (0)

#define HC_CHECK_LAUNCH()         \
    do {                          \
        ::hc::count_launch();     \
        HC_CUDA(cudaGetLastError()); \
    } while (0)

#define HC_REQUIRE(cond, ...)                                \
    do {                                                     \
        if (!(cond)) HC_FAIL(HC_ERR_INVALID, __VA_ARGS__);   \
    } while (0)

#define HC_TRY(expr)                    \
    do {                                \
        hc_status s_ = (expr);          \
        if (s_ != HC_OK) return s_;     \
    } while (0)

// Device allocation that only grows; freed by the owner's destructor.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    hc_status ensure(size_t need) {
        if (need <= bytes) return HC_OK;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        if (need == 0) return HC_OK;
        cudaError_t e = cudaMalloc(&ptr, need);
        if (e != cudaSuccess) {
            ptr = nullptr;
            HC_FAIL(HC_ERR_ALLOC, "cudaMalloc(%zu) failed: %s", need, cudaGetErrorString(e));
        }
        bytes = need;
        return HC_OK;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return reinterpret_cast<T*>(ptr); }
};

template <class T>
hc_status upload(DevBuf& b, const T* host, size_t count) {
    HC_TRY(b.ensure(count * sizeof(T)));
    if (count) HC_CUDA(cudaMemcpy(b.ptr, host, count * sizeof(T), cudaMemcpyHostToDevice));
    return HC_OK;
}

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace hc
