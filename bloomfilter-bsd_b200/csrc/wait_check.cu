// wait_check.cu -- the bounded device waits give up and report, without a fault.
//
// Two kernels of this library wait on words that other CTAs write: the
// decoupled look-back of the ordered compaction (a tile waits for its
// predecessors' status words) and the batched kernel's item dependencies (an
// item waits for a per-filter counter).  Each wait spins a bounded number of
// times, then sets an error bit, stops waiting and lets the kernel finish, so
// the host sees DTLG_ERR_TIMEOUT and the context stays usable.  In a correct
// run nothing makes those waits run out; dtlg_check_wait_timeout runs the same
// two wait loops against words that nothing ever sets, with a short limit, so
// a test can see that they end and report.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/dtlg.h"
#include "batched.cuh"
#include "status.hpp"

namespace {

using namespace dtlg;

// One CTA.  Warp 0 looks back from tile 40 over 40 status words that stay
// zero (no predecessor ever publishes); then the CTA waits for a counter
// that stays zero.
__global__ void __launch_bounds__(kProbeThreads) wait_timeout_kernel(unsigned long long* status, unsigned int* err,
                                                                     const unsigned int* ctr, uint32_t limit,
                                                                     unsigned int* prefix_out) {
  ProbeArgs a{};
  a.status = status;
  a.err = err;
  if (threadIdx.x < 32) {
    const uint32_t excl = look_back(a, 40, threadIdx.x, limit);
    if (threadIdx.x == 0) *prefix_out = excl;
  }
  __syncthreads();
  wait_counter(ctr, 1, err, limit);
}

}  // namespace

extern "C" dtlg_status dtlg_check_wait_timeout(uint32_t spin_limit, uint32_t* err_bits) {
  if (!err_bits) return DTLG_ERR_NULL;
  if (spin_limit == 0 || spin_limit > kSpinLimit) return DTLG_ERR_INVALID_CONFIG;
  // 40 status words, the error word, the counter and the returned prefix
  constexpr size_t kBytes = 40 * 8 + 16;
  void* buf = nullptr;
  DTLG_TRY_CUDA(cudaMalloc(&buf, kBytes));
  cudaError_t e = cudaMemset(buf, 0, kBytes);
  unsigned long long* status = static_cast<unsigned long long*>(buf);
  unsigned int* tail = reinterpret_cast<unsigned int*>(status + 40);
  if (e == cudaSuccess) {
    wait_timeout_kernel<<<1, kProbeThreads>>>(status, tail, tail + 1, spin_limit, tail + 2);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  unsigned int host[3] = {0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(host, tail, sizeof(host), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) return cuda_error_status(e);
  *err_bits = host[0];
  return DTLG_OK;
}
