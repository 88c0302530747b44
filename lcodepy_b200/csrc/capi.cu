// Error reporting, version and launch accounting for the C ABI.
#include <atomic>
#include <cstdarg>
#include <cstring>

#include "common.cuh"

namespace lcb {

static thread_local char g_err[512] = "";
static std::atomic<int64_t> g_launches{0};

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return LCB_OK;
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return LCB_ERR_CUDA;
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int sm_count()
{
    static int cached = 0;
    if (cached == 0) {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0)
            cached = n;
        else
            cached = 148;
    }
    return cached;
}

}  // namespace lcb

extern "C" const char *lcb_last_error(void) { return lcb::g_err; }
extern "C" int lcb_version(void) { return 100; }
extern "C" int64_t lcb_launch_count(void) { return lcb::g_launches.load(); }
