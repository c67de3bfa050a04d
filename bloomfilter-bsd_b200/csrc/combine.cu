// combine.cu -- OR-combines partial Bloom filters (sharded builds), and
// copies filter words between devices (per-device replicas).
//
// A Bloom build sharded over G GPUs inserts each GPU's share of the keys into
// its own copy of the filter words; OR is the only reduction the words need,
// and NCCL has none, so the combine step exchanges word ranges (all-to-all),
// ORs them here and gathers the result.  The reference's counterpart is its
// per-NUMA-node replication (filter.hpp:128-152), which copies a finished
// filter instead of building shards.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/dtlg.h"
#include "status.hpp"

namespace {

// dst[i] |= src[j * stride + i] for j < n_src (grid-stride, coalesced).
__global__ void __launch_bounds__(256) or_words_kernel(uint64_t* __restrict__ dst, const uint64_t* __restrict__ src,
                                                       uint64_t n, uint32_t n_src, uint64_t stride) {
  for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * 256) {
    uint64_t v = dst[i];
    for (uint32_t j = 0; j < n_src; j++) v |= __ldcs(src + j * stride + i);
    dst[i] = v;
  }
}

}  // namespace

extern "C" {

dtlg_status dtlg_or_words(uint64_t* dst, const uint64_t* src, uint64_t n_words, uint32_t n_src, uint64_t src_stride,
                          dtlg_stream_t stream) {
  if (n_words == 0 || n_src == 0) return DTLG_OK;
  if (!dst || !src) return DTLG_ERR_NULL;
  if (n_src > 1 && src_stride < n_words) return DTLG_ERR_INVALID_CONFIG;
  int dev = 0, sms = 0;
  DTLG_TRY_CUDA(cudaGetDevice(&dev));
  DTLG_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint64_t blocks = (n_words + 255) / 256;
  const unsigned grid = static_cast<unsigned>(blocks < static_cast<uint64_t>(sms) * 8 ? blocks : sms * 8ull);
  or_words_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(dst, src, n_words, n_src, src_stride);
  DTLG_TRY_CUDA(cudaGetLastError());
  return DTLG_OK;
}

// A copy engine transfer (cudaMemcpyPeerAsync): no kernel of this library or
// of any other reads the other device's memory.
dtlg_status dtlg_copy_words_peer(uint64_t* dst, int dst_device, const uint64_t* src, int src_device,
                                 uint64_t n_words, dtlg_stream_t stream) {
  if (n_words == 0) return DTLG_OK;
  if (!dst || !src) return DTLG_ERR_NULL;
  if (dst_device < 0 || src_device < 0) return DTLG_ERR_INVALID_CONFIG;
  DTLG_TRY_CUDA(cudaMemcpyPeerAsync(dst, dst_device, src, src_device, n_words * sizeof(uint64_t),
                                    reinterpret_cast<cudaStream_t>(stream)));
  return DTLG_OK;
}

}  // extern "C"
