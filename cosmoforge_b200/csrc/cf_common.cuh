// Shared definitions for the cosmoforge_b200 device library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define CF_OK 0
#define CF_ERR_ARG -1
#define CF_ERR_CUDA -2
#define CF_ERR_TIMEOUT -3
#define CF_ERR_UNSUPPORTED -4
#define CF_ERR_TOO_LARGE -5

#define CF_PI 3.14159265358979323846

// Number of kernels this library has launched (host-side count, read by
// cf_launch_count); every launch site goes through CF_CHECK_LAUNCH.
extern unsigned long long g_cf_launch_count;

// Count the launch and return CF_ERR_CUDA from the enclosing function if it failed.
#define CF_CHECK_LAUNCH()                                  \
    do {                                                   \
        ++g_cf_launch_count;                               \
        cudaError_t e_ = cudaGetLastError();               \
        if (e_ != cudaSuccess) return CF_ERR_CUDA;         \
    } while (0)

#define CF_CHECK(call)                                     \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return CF_ERR_CUDA;         \
    } while (0)

static inline int cf_cdiv(long a, long b) { return (int)((a + b - 1) / b); }

#ifdef __CUDACC__
#include <cuda_bf16.h>
// Next BF16 split plane of x (round to nearest), and x minus it (exact in FP64).
__device__ __forceinline__ __nv_bfloat16 cf_bf16_plane(double& x)
{
    const __nv_bfloat16 h = __double2bfloat16(x);
    x -= (double)__bfloat162float(h);
    return h;
}
#endif

#ifdef __cplusplus
#include <atomic>

#define CF_MAX_DEVICES 64

// Opt `kernel` in to `bytes` of dynamic shared memory on the calling thread's
// current device.  cudaFuncSetAttribute acts on the current device only, so
// each call site keeps one flag per device (`done`, a zero-initialised static
// array of CF_MAX_DEVICES); two host threads that race on a device's first
// call both set the attribute, which is idempotent.  Devices past the table
// set it on every call.
template <typename K>
static inline int cf_smem_optin(K* kernel, int bytes, std::atomic<int>* done)
{
    int dev = -1;
    CF_CHECK(cudaGetDevice(&dev));
    const bool tracked = dev >= 0 && dev < CF_MAX_DEVICES;
    if (tracked && done[dev].load(std::memory_order_acquire)) return CF_OK;
    CF_CHECK(cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (tracked) done[dev].store(1, std::memory_order_release);
    return CF_OK;
}
#endif
