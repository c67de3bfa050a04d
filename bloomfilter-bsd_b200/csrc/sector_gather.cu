// sector_gather.cu -- the random-sector gather rate of this GPU, the roofline
// of probes whose filter stays in L2.
//
// A probe of an L2-resident filter moves no filter bytes from HBM: what bounds
// it is how many random 32-byte sectors the SMs can gather from L2 per second.
// That rate is a property of the GPU, the buffer size and the load
// instruction, so it is measured here with the probe's own load (one 256-bit
// read-only load per sector) and no other work: n random sectors of a caller
// buffer, several independent loads in flight per thread, every loaded word
// folded into one XOR so that nothing is optimised away.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/dtlg.h"
#include "status.hpp"

namespace {

constexpr int kGatherThreads = 256;
constexpr int kGatherUnroll = 4;  // independent loads in flight per thread

// sector i of the stream: a multiplicative hash of i scaled to [0, rows)
__host__ __device__ inline uint32_t gather_row(uint64_t i, uint32_t rows) {
  uint64_t x = (i + 1) * 0x9e3779b97f4a7c15ull;
  x ^= x >> 29;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 32;
  return static_cast<uint32_t>(((x & 0xffffffffull) * rows) >> 32);
}

__global__ void __launch_bounds__(kGatherThreads) sector_gather_kernel(const uint64_t* __restrict__ buf,
                                                                      uint32_t rows, uint64_t n,
                                                                      unsigned long long* sink) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * kGatherThreads;
  unsigned long long acc = 0;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(kGatherThreads) + threadIdx.x; i < n;
       i += stride * kGatherUnroll) {
    unsigned long long v[kGatherUnroll][4];
#pragma unroll
    for (int u = 0; u < kGatherUnroll; u++) {
      const uint64_t j = i + u * stride;
      if (j < n) {
        const uint64_t* p = buf + static_cast<uint64_t>(gather_row(j, rows)) * 4;
        asm volatile("ld.global.nc.v4.u64 {%0,%1,%2,%3}, [%4];"
                     : "=l"(v[u][0]), "=l"(v[u][1]), "=l"(v[u][2]), "=l"(v[u][3])
                     : "l"(p));
      } else {
        v[u][0] = v[u][1] = v[u][2] = v[u][3] = 0;
      }
    }
#pragma unroll
    for (int u = 0; u < kGatherUnroll; u++) acc ^= v[u][0] ^ (v[u][1] * 3) ^ (v[u][2] * 5) ^ (v[u][3] * 7);
  }
  atomicXor(sink, acc);
}

}  // namespace

extern "C" {

dtlg_status dtlg_sector_gather(const uint64_t* buf, uint64_t bytes, uint64_t n_sectors, uint64_t* sink_dev,
                               dtlg_stream_t stream) {
  if (n_sectors == 0) return DTLG_OK;
  if (!buf || !sink_dev) return DTLG_ERR_NULL;
  if (reinterpret_cast<uintptr_t>(buf) & 31u) return DTLG_ERR_ALIGNMENT;
  const uint64_t rows = bytes / 32;
  if (rows == 0 || rows > 0xffffffffull) return DTLG_ERR_INVALID_CONFIG;
  int dev = 0, sms = 0, occ = 0;
  DTLG_TRY_CUDA(cudaGetDevice(&dev));
  DTLG_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DTLG_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sector_gather_kernel, kGatherThreads, 0));
  const uint64_t need = (n_sectors + kGatherThreads - 1) / kGatherThreads;
  const uint64_t full = static_cast<uint64_t>(sms) * (occ > 0 ? occ : 1);
  const unsigned grid = static_cast<unsigned>(need < full ? need : full);
  sector_gather_kernel<<<grid, kGatherThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      buf, static_cast<uint32_t>(rows), n_sectors, reinterpret_cast<unsigned long long*>(sink_dev));
  DTLG_TRY_CUDA(cudaGetLastError());
  return DTLG_OK;
}

}  // extern "C"
