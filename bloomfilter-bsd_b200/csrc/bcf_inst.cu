// bcf_inst.cu -- compiled blocked cuckoo kernels for every tag size /
// associativity the reference's dispatcher accepts (blocked_cuckoofilter.hpp:
// 270-297; the block size is a run-time parameter of the kernels), and the
// classic Bloom filter's kernels (k is a run-time parameter).
#include "registry.hpp"

namespace dtlg {
namespace {

// bloomfilter_logic.hpp:94-121: k word ORs per key; OR is order-independent,
// so the words equal a sequential build's.
__global__ void __launch_bounds__(256) classic_build_kernel(const __grid_constant__ ClassicBuildArgs a) {
  for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < a.n_phys;
       p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    if (p < a.pre) continue;
    const uint32_t key = __ldg(a.keys_al + p);
#pragma unroll
    for (uint32_t i = 0; i < kClassicMaxK; i++) {
      if (i >= a.k) break;
      const uint32_t h = key * mul_const(static_cast<int>(i));
      atomicOr(a.filter + block_index(h, a.addr), 1u << ((h >> a.bit_shift) & a.bit_mask));
    }
  }
}

cudaError_t classic_build(const ClassicBuildArgs& a, int grid, cudaStream_t s) {
  classic_build_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// The classic Bloom filter's k words lie anywhere in the filter: no
// partitioned plan; small filters take the shared-memory plan.
ClassicKernels classic_entry() { return ClassicKernels{probe_entry<ClassicOps, false, true>(), &classic_build}; }

struct RegBcf {
  RegBcf() {
    register_bcf(bcf_entry<8, 4>());
    register_bcf(bcf_entry<8, 8>());
    register_bcf(bcf_entry<10, 6>());
    register_bcf(bcf_entry<12, 4>());
    register_bcf(bcf_entry<16, 2>());
    register_bcf(bcf_entry<16, 4>());
    register_classic(classic_entry());
  }
} reg_bcf;
}  // namespace
}  // namespace dtlg
