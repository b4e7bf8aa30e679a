// Shared definitions for the cosmoforge_b200 device library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define CF_OK 0
#define CF_ERR_ARG -1
#define CF_ERR_CUDA -2
#define CF_ERR_TIMEOUT -3
#define CF_ERR_UNSUPPORTED -4

#define CF_PI 3.14159265358979323846

// Return CF_ERR_CUDA from the enclosing function if the last launch failed.
#define CF_CHECK_LAUNCH()                                  \
    do {                                                   \
        cudaError_t e_ = cudaGetLastError();               \
        if (e_ != cudaSuccess) return CF_ERR_CUDA;         \
    } while (0)

#define CF_CHECK(call)                                     \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return CF_ERR_CUDA;         \
    } while (0)

static inline int cf_cdiv(long a, long b) { return (int)((a + b - 1) / b); }
