// Error reporting for the C ABI.
#include <atomic>

#include "hc_common.cuh"

namespace hc {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

}  // namespace hc

extern "C" const char* hc_last_error(void) { return hc::g_last_error.c_str(); }
extern "C" const char* hc_version(void) { return "hc-b200 0.1 (sm_100a)"; }
extern "C" int64_t hc_kernel_launches(void) { return hc::g_launches.load(std::memory_order_relaxed); }
