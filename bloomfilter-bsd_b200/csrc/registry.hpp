// registry.hpp -- table of compiled kernel instantiations, keyed by config.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bcf.cuh"
#include "bloom.cuh"
#include "classic.cuh"
#include "cuckoo.cuh"
#include "probe.cuh"
#include "probe2.cuh"
#include "probe3.cuh"

namespace dtlg {

using probe_fn = cudaError_t (*)(const ProbeArgs&, int grid, cudaStream_t);
using build_fn = cudaError_t (*)(const BuildArgs&, int grid, cudaStream_t);
using occ_fn = int (*)();
using probe_bits_fn = cudaError_t (*)(const ProbeArgs&, uint32_t* bits, int or_into, int grid, cudaStream_t);

// Register-budget variants of probe_bits_kernel: 0 = 8 CTAs/SM (32 registers),
// 1 = 4 CTAs/SM (64 registers, more filter loads in flight per thread).
constexpr int kBitsVariants = 2;
using pairs_fn = cudaError_t (*)(const PairsArgs&, int grid, cudaStream_t);
// plan 4: bitmask probe against a shared-memory copy of a filter of words32
// 32-bit words; chunks = 128-key chunks of the batch, sms = SM count
using smem_fn = cudaError_t (*)(const ProbeArgs&, uint32_t* bits, uint32_t words32, uint64_t chunks, int sms,
                                cudaStream_t);

// The probe kernels every filter kind provides to the probe plans.
struct ProbeKernels {
  probe_fn probe;                               // plan 1: fused probe + compaction
  occ_fn probe_blocks_per_sm;
  probe_bits_fn probe_bits[kBitsVariants];      // plan 2: match bitmask
  occ_fn bits_blocks_per_sm[kBitsVariants];
  pairs_fn probe_pairs[kBitsVariants];          // plan 3: partitioned (null: not offered)
  occ_fn pairs_blocks_per_sm[kBitsVariants];
  smem_fn probe_smem;                           // plan 4: filter in shared memory (null: not offered)
  occ_fn bits_local_bytes[kBitsVariants];       // register spills per thread of each variant
  occ_fn pairs_local_bytes[kBitsVariants];
};

struct BloomKernels {
  uint32_t word_bytes, w, s, z, k;
  ProbeKernels pk;
  build_fn build;
  // build from range-grouped (key, position) pairs
  cudaError_t (*build_pairs)(const PartArgs& part, void* filter, const Addr& addr, int grid, cudaStream_t);
};

struct CuckooKernels {
  uint32_t t, b;
  ProbeKernels pk;
  void (*unpack)(const uint32_t* table, uint32_t* slots, uint32_t buckets, int grid, cudaStream_t);
  void (*insert)(const CuckooBuildArgs&, int grid, cudaStream_t);
  void (*pack)(uint32_t* table, const uint32_t* slots, uint32_t buckets, uint64_t words, int grid,
               cudaStream_t);
  void (*count)(const uint32_t* table, uint32_t buckets, uint64_t victim_word, unsigned long long* out,
                int grid, cudaStream_t);
};

struct BcfKernels {
  uint32_t t, a;
  ProbeKernels pk;
  cudaError_t (*insert)(const BcfBuildArgs&, int grid, cudaStream_t);
  // insert from range-grouped (key, position) pairs
  cudaError_t (*insert_pairs)(const BcfBuildArgs&, const PartArgs& part, int grid, cudaStream_t);
};

struct ClassicKernels {
  ProbeKernels pk;
  cudaError_t (*build)(const ClassicBuildArgs&, int grid, cudaStream_t);
};

void register_bloom(const BloomKernels& k);
void register_cuckoo(const CuckooKernels& k);
void register_bcf(const BcfKernels& k);
const BcfKernels* find_bcf(uint32_t t, uint32_t a);
void register_classic(const ClassicKernels& k);
const ClassicKernels* find_classic();
const BloomKernels* find_bloom(uint32_t word_bytes, uint32_t w, uint32_t s, uint32_t z, uint32_t k);
const CuckooKernels* find_cuckoo(uint32_t t, uint32_t b);
int registered_bloom_count();

// Keys per probe tile: 256 threads x 4 keys x kProbeRounds.
constexpr int kProbeRounds = 4;
constexpr uint32_t kProbeTile = kProbeThreads * 4 * kProbeRounds;

#ifdef __CUDACC__
template <class Ops, int MINB>
struct BitsLaunch {
  static cudaError_t run(const ProbeArgs& a, uint32_t* bits, int or_into, int grid, cudaStream_t s) {
    probe_bits_kernel<Ops, MINB><<<grid, 256, 0, s>>>(a, bits, or_into);
    return cudaGetLastError();
  }
  static int occupancy() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, probe_bits_kernel<Ops, MINB>, 256, 0);
    return n;
  }
  static int local_bytes() {
    static const int v = local_bytes_of(probe_bits_kernel<Ops, MINB>);
    return v;
  }
};

// Local memory of a kernel per thread (register spills; none of these
// kernels has a stack otherwise), -1 if the query fails.
template <class K>
int local_bytes_of(K kernel) {
  cudaFuncAttributes at{};
  return cudaFuncGetAttributes(&at, kernel) == cudaSuccess ? static_cast<int>(at.localSizeBytes) : -1;
}

template <class Ops, int MINB>
struct PairsLaunch {
  // the pair probe, then the keys of overflowing runs (returns at once when none)
  static cudaError_t run(const PairsArgs& a, int grid, cudaStream_t s) {
    probe_pairs_kernel<Ops, MINB><<<grid, 256, 0, s>>>(a);
    probe_overflow_kernel<Ops><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
  }
  static int occupancy() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, probe_pairs_kernel<Ops, MINB>, 256, 0);
    return n;
  }
  static int local_bytes() {
    static const int v = local_bytes_of(probe_pairs_kernel<Ops, MINB>);
    return v;
  }
};

template <class Ops>
struct FusedLaunch {
  static cudaError_t run(const ProbeArgs& a, int grid, cudaStream_t s) {
    probe_kernel<Ops, kProbeRounds><<<grid, kProbeThreads, 0, s>>>(a);
    return cudaGetLastError();
  }
  static int occupancy() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, probe_kernel<Ops, kProbeRounds>, kProbeThreads, 0);
    return n;
  }
};

template <class Cfg>
struct BloomLaunch {
  static cudaError_t build(const BuildArgs& a, int grid, cudaStream_t s) {
    bloom_build_kernel<Cfg><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t build_pairs(const PartArgs& part, void* filter, const Addr& addr, int grid, cudaStream_t s) {
    bloom_build_pairs_kernel<Cfg><<<grid, 256, 0, s>>>(part, filter, addr);
    return cudaGetLastError();
  }
};

template <class Ops>
struct SmemLaunch {
  static cudaError_t run(const ProbeArgs& a, uint32_t* bits, uint32_t words32, uint64_t chunks, int sms,
                         cudaStream_t s) {
    static const cudaError_t attr = [] {
      int dev = 0, optin = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(probe_smem_kernel<Ops>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
      return e;
    }();
    if (attr != cudaSuccess) return attr;
    const size_t bytes = (static_cast<size_t>(words32) * 4 + 15) & ~static_cast<size_t>(15);
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, probe_smem_kernel<Ops>, kSmemThreads, bytes);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    // one chunk per warp at most; at most the resident CTAs (each copies the filter)
    const uint64_t want = (chunks + kSmemThreads / 32 - 1) / (kSmemThreads / 32);
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(want, static_cast<uint64_t>(sms) * occ)));
    probe_smem_kernel<Ops><<<grid, kSmemThreads, bytes, s>>>(a, bits, words32);
    return cudaGetLastError();
  }
};

// Probe kernels of one Ops type; Pairs = false leaves the partitioned plan
// out, Smem = false the shared-memory plan.
template <class Ops, bool Pairs, bool Smem = false>
ProbeKernels probe_entry() {
  using F = FusedLaunch<Ops>;
  using B8 = BitsLaunch<Ops, 8>;
  using B4 = BitsLaunch<Ops, 4>;
  using P8 = PairsLaunch<Ops, 8>;
  using P4 = PairsLaunch<Ops, 4>;
  ProbeKernels k{&F::run, &F::occupancy, {&B8::run, &B4::run}, {&B8::occupancy, &B4::occupancy},
                 {nullptr, nullptr}, {nullptr, nullptr}, nullptr, {&B8::local_bytes, &B4::local_bytes},
                 {nullptr, nullptr}};
  if constexpr (Smem) k.probe_smem = &SmemLaunch<Ops>::run;
  if constexpr (Pairs) {
    k.probe_pairs[0] = &P8::run;
    k.probe_pairs[1] = &P4::run;
    k.pairs_blocks_per_sm[0] = &P8::occupancy;
    k.pairs_blocks_per_sm[1] = &P4::occupancy;
    k.pairs_local_bytes[0] = &P8::local_bytes;
    k.pairs_local_bytes[1] = &P4::local_bytes;
  }
  return k;
}

template <typename Word, int W, int S, int Z, int K>
BloomKernels bloom_entry() {
  using C = BloomCfg<Word, W, S, Z, K>;
  return BloomKernels{static_cast<uint32_t>(sizeof(Word)), W, S, Z, K, probe_entry<BloomOps<C>, true, true>(),
                      &BloomLaunch<C>::build, &BloomLaunch<C>::build_pairs};
}

template <int T, int B>
struct CuckooLaunch {
  using C = CuckooCfg<T, B>;
  static void unpack(const uint32_t* t, uint32_t* sl, uint32_t nb, int grid, cudaStream_t s) {
    cuckoo_unpack_kernel<C><<<grid, 256, 0, s>>>(t, sl, nb);
  }
  static void insert(const CuckooBuildArgs& a, int grid, cudaStream_t s) {
    cuckoo_insert_kernel<C><<<grid, 256, 0, s>>>(a);
  }
  static void pack(uint32_t* t, const uint32_t* sl, uint32_t nb, uint64_t words, int grid, cudaStream_t s) {
    cuckoo_pack_kernel<C><<<grid, 256, 0, s>>>(t, sl, nb, words);
  }
  static void count(const uint32_t* t, uint32_t nb, uint64_t vw, unsigned long long* out, int grid,
                    cudaStream_t s) {
    cuckoo_count_kernel<C><<<grid, 256, 0, s>>>(t, nb, vw, out);
  }
};

// Cuckoo buckets are probed in bucket-range passes, not partitioned: a key's
// two buckets lie anywhere in the table.
template <int T, int B>
CuckooKernels cuckoo_entry() {
  using L = CuckooLaunch<T, B>;
  return CuckooKernels{T, B, probe_entry<CuckooOps<CuckooCfg<T, B>>, false>(), &L::unpack, &L::insert, &L::pack,
                       &L::count};
}

template <int T, int A>
struct BcfLaunch {
  static cudaError_t insert(const BcfBuildArgs& a, int grid, cudaStream_t s) {
    bcf_insert_kernel<BcfCfg<T, A>><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t insert_pairs(const BcfBuildArgs& a, const PartArgs& part, int grid, cudaStream_t s) {
    bcf_insert_pairs_kernel<BcfCfg<T, A>><<<grid, 256, 0, s>>>(a, part);
    return cudaGetLastError();
  }
};

template <int T, int A>
BcfKernels bcf_entry() {
  return BcfKernels{T, A, probe_entry<BcfOps<BcfCfg<T, A>>, true>(), &BcfLaunch<T, A>::insert,
                    &BcfLaunch<T, A>::insert_pairs};
}
#endif

}  // namespace dtlg
