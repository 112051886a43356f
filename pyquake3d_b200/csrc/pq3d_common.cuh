// Shared definitions for the pq3d CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Status codes returned by every pq3d_* entry point (0 = success).
#define PQ3D_OK 0
#define PQ3D_ERR_ARG -1        // bad argument (null pointer, size out of range)
#define PQ3D_ERR_CUDA -2       // a CUDA runtime call failed
#define PQ3D_ERR_RANK -3       // ACA rank cap reached (block must fall back to dense)
#define PQ3D_ERR_DT -4         // step-size controller gave up (h < 1e-15 or > 20 rejects)
#define PQ3D_ERR_TIMEOUT -5    // a bounded device-side wait ran out
#define PQ3D_ERR_NOMEM -6      // scratch too small

#define PQ3D_CHECK(call)                                   \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return PQ3D_ERR_CUDA;       \
    } while (0)

static inline int pq3d_launch_status()
{
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PQ3D_OK : PQ3D_ERR_CUDA;
}

#define PQ3D_EXPORT extern "C" __attribute__((visibility("default")))
