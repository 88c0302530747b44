// Shared device helpers for liblcb (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <atomic>

#include "../../include/lcb.h"

namespace lcb {

// ---- error reporting (host) ----
void set_error(const char *fmt, ...);
int cuda_check(cudaError_t e, const char *what);
void count_launch(int n = 1);

#define LCB_LAUNCH_CHECK(what)                                              \
    do {                                                                    \
        ::lcb::count_launch();                                              \
        cudaError_t _e = cudaGetLastError();                                \
        if (_e != cudaSuccess) return ::lcb::cuda_check(_e, what);          \
    } while (0)

#define LCB_REQUIRE(cond, ...)                                              \
    do {                                                                    \
        if (!(cond)) { ::lcb::set_error(__VA_ARGS__); return LCB_ERR_INVALID; } \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// One-time opt-in of a kernel to `bytes` of dynamic shared memory on the
// current device; `done` remembers the devices already set (the attribute is
// per device, so a process that uses several GPUs sets it on each).  Host
// threads driving different GPUs may call this at once: the mask is atomic,
// and setting the attribute twice for one device is harmless.
template <typename K>
inline cudaError_t ensure_smem(K kernel, size_t bytes, std::atomic<unsigned long long> &done)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? (1ull << dev) : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// ---- programmatic dependent launch ----
// A kernel launched with launch_after() may be scheduled while its
// predecessor in the stream is still running; it must call pdl_wait() before
// its first global memory access (read or write), which returns once the
// predecessor has completed and its writes are visible.  pdl_trigger() lets
// the successor be scheduled early.  Both are no-ops for ordinary launches.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_after(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                cudaStream_t st, Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args &&>(args)...);
}

// Number of SMs of the current device (cached per process; one device per
// process is the deployment model).
int sm_count();

// ---- 4th-order spline weights at offsets -2..2 ----
// The reference's weight4 (lcode/plasma3d/weights.py:13-31, :127-148),
// evaluated for all five offsets at once.
// Divisions by 6 and 24 are multiplications by the rounded reciprocals here
// (at most an ulp from the reference's quotients; IEEE division would cost a
// Newton sequence per term).
__device__ __forceinline__ void weights4(double x, double w[5])
{
    constexpr double r6 = 1.0 / 6.0, r24 = 1.0 / 24.0;
    const double x2 = x * x, x3 = x2 * x, x4 = x3 * x;
    const double a = 0.5 - x, b = 0.5 + x;
    w[0] = a * a * a * a * r24;
    w[1] = 19 / 96. - 11 / 24. * x + x2 * 0.25 + x3 * r6 - x4 * r6;
    w[2] = 115 / 192. - 5 / 8. * x2 + x4 * 0.25;
    w[3] = 19 / 96. + 11 / 24. * x + x2 * 0.25 - x3 * r6 - x4 * r6;
    w[4] = b * b * b * b * r24;
}

// Cell of a position (in cell units, already offset by +0.5) and the local
// coordinate in [-0.5, 0.5): the reference's
//   x_loc = x_h - floor(x_h) - 0.5;  ix = floor(x_h) + floor(N / 2).
__device__ __forceinline__ int cell_of(double x_h, int half_n, double &loc)
{
    const double f = floor(x_h);
    loc = x_h - f - 0.5;
    // Values far outside the grid (or NaN) must not overflow the int cast;
    // clamp to a sentinel the caller's bounds check rejects.
    if (!(f > -1e9 && f < 1e9)) return INT32_MIN / 2;
    return (int)f + half_n;
}

}  // namespace lcb
