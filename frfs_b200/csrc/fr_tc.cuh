// Internal interface of the tensor-core FR right-hand side.
#pragma once
#include <cuda_runtime.h>

#include "../../include/bdgfs.h"

namespace bdgfs {

// bdgfs_fr_rhs on the tensor cores; BDGFS_EUNSUPPORTED (nothing launched)
// for FP64 state, el.engine != 1 or an element shape without a variant.
int fr_rhs_tc(const bdgfs_fr_eles& el, const bdgfs_fr_walls& wl, const void* u, const void* uf, void* out,
              double a, double b, const void* x1, double c1, const void* x2, double c2, cudaStream_t st);

}  // namespace bdgfs
