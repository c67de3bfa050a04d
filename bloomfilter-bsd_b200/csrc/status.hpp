// status.hpp -- CUDA error reporting shared by the translation units of libdtlg.so.
#pragma once

#include <cuda_runtime.h>

#include "../../include/dtlg.h"

namespace dtlg {
// Records cudaGetErrorString(e) for dtlg_last_cuda_error(); returns DTLG_ERR_CUDA.
dtlg_status cuda_error_status(cudaError_t e);
}  // namespace dtlg

#define DTLG_TRY_CUDA(x)                                             \
  do {                                                               \
    cudaError_t _e = (x);                                            \
    if (_e != cudaSuccess) return ::dtlg::cuda_error_status(_e);     \
  } while (0)
