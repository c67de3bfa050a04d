// classic.cuh -- classic Bloom filter probe and build.
//
// Reference: bloomfilter/bloomfilter_logic.hpp:22-212 (experimental in the
// reference: no dispatcher, no filter_base wrapper).  The filter is an array
// of 32-bit words, each its own addressing "block"; key x sets / tests one bit
// in each of k words:
//
//   h_i  = x * C[i]                  (dyn::mul32, hash_family.hpp:271-299; i < k <= 17)
//   word = addr(h_i)                 (POW2 top bits or MAGIC fast mod of h_i)
//   bit  = (h_i >> (27 - log2 B)) & 31                      (:105,138)
//
// The bit shift is undefined C++ once log2 B > 27 (POW2) and for MAGIC (whose
// addressing bits are 32); the reference as compiled (g++ 13, x86-64, -O2)
// takes a POW2 shift count mod 32 and folds the MAGIC bit index to 0, and so
// does this kernel (bit = (h >> bit_shift) & bit_mask, both set on the host).
// contains stops at the first clear bit, as the reference does (:139-141).
#pragma once

#include <cstdint>

#include "common.cuh"
#include "probe.cuh"

namespace dtlg {

constexpr uint32_t kClassicMaxK = 17;  // hash functions C[0..16]

struct ClassicBuildArgs {
  uint32_t* filter;
  const uint32_t* keys_al;
  uint64_t n_phys;
  uint32_t pre;
  Addr addr;
  uint32_t k, bit_shift, bit_mask;
};

#ifdef __CUDACC__

struct ClassicOps {
  __device__ __forceinline__ static bool contains(const ProbeArgs& a, uint32_t key) {
    const unsigned int* w = static_cast<const unsigned int*>(a.filter);
    bool hit = true;
#pragma unroll
    for (uint32_t i = 0; i < kClassicMaxK; i++) {
      if (i >= a.cbf_k || !hit) break;
      const uint32_t h = key * mul_const(static_cast<int>(i));
      const uint32_t bit = (h >> a.cbf_bit_shift) & a.cbf_bit_mask;
      hit = (__ldg(w + block_index(h, a.addr)) >> bit) & 1u;
    }
    return hit;
  }

  // The same test against a copy of the filter in shared memory (plan 4).
  __device__ __forceinline__ static bool contains_shared(const void* sfilter, const ProbeArgs& a, uint32_t key) {
    const unsigned int* w = static_cast<const unsigned int*>(sfilter);
    bool hit = true;
#pragma unroll
    for (uint32_t i = 0; i < kClassicMaxK; i++) {
      if (i >= a.cbf_k || !hit) break;
      const uint32_t h = key * mul_const(static_cast<int>(i));
      const uint32_t bit = (h >> a.cbf_bit_shift) & a.cbf_bit_mask;
      hit = (w[block_index(h, a.addr)] >> bit) & 1u;
    }
    return hit;
  }
};

#endif  // __CUDACC__

}  // namespace dtlg
