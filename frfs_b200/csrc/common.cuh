// Shared definitions for the bdgfs CUDA kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/bdgfs.h"

namespace bdgfs {

// Map a CUDA error to the library status code.
static inline int cuda_status(cudaError_t e)
{
    return e == cudaSuccess ? BDGFS_OK : BDGFS_ECUDA;
}

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Block-wide sum of NV doubles; every thread gets the result.
// red must hold NV * (blockDim.x / 32) doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarp = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = v[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[j] = x;
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) red[warp * NV + j] = v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double s = 0.0;
        for (int w = 0; w < nwarp; ++w) s += red[w * NV + j];
        v[j] = s;
    }
    __syncthreads();
}

}  // namespace bdgfs
