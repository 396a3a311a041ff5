// Internal interface between the GEMM entry point and its engines.
#pragma once
#include <cuda_runtime.h>

#include "../../include/bdgfs.h"

namespace bdgfs {

// Persistent, TMA-fed, warp-specialised tcgen05 GEMM for bf16 operands whose
// K index is contiguous.  Returns BDGFS_EUNSUPPORTED (launching nothing)
// when the operands do not qualify; the caller then uses the general engine.
int tma_gemm(const bdgfs_gemm_args& g, cudaStream_t st);

}  // namespace bdgfs
