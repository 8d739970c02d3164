// api.cu -- library-wide C-ABI plumbing: error reporting, launch accounting,
// device properties.
#include <stdarg.h>

#include <atomic>

#include "common.cuh"

namespace tchll {

static thread_local char g_err[1024] = "";
static std::atomic<uint64_t> g_launches{0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t e, const char* what) {
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return TCHLL_ECUDA;
}

void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
    if (dev < 64 && cached[dev]) return cached[dev];
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    if (dev < 64) cached[dev] = n;
    return n;
}

}  // namespace tchll

TCHLL_EXPORT const char* tchll_last_error(void) { return tchll::g_err; }

TCHLL_EXPORT int tchll_version(void) { return 10000; }

TCHLL_EXPORT uint64_t tchll_launch_count(void) { return tchll::g_launches.load(std::memory_order_relaxed); }
