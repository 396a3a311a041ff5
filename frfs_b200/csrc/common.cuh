// Shared definitions for the bdgfs CUDA kernels.
#pragma once
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>
#include <cuda_runtime.h>

#include "../../include/bdgfs.h"

namespace bdgfs {

// Map a CUDA error to the library status code.
static inline int cuda_status(cudaError_t e)
{
    return e == cudaSuccess ? BDGFS_OK : BDGFS_ECUDA;
}

// Largest device ordinal the per-device records cover.
constexpr int kMaxDevices = 64;

// Dynamic shared-memory opt-in of kernel `func` on the current device.  The
// attribute belongs to one (kernel, device) pair, so the record is kept per
// pair (the largest size opted in); the attribute is set only when a size
// above that record is asked for, so that calls made during CUDA-graph
// capture issue no attribute change.  Sizes up to 48 KB need no opt-in.
// Thread-safe.
static inline int smem_optin(const void* func, size_t smem)
{
    if (smem <= 48 * 1024) return BDGFS_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BDGFS_ECUDA;
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = done[{func, dev}];
    if (smem <= have) return BDGFS_OK;
    if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return BDGFS_ECUDA;
    have = smem;
    return BDGFS_OK;
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
