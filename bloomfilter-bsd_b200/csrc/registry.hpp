// registry.hpp -- table of compiled kernel instantiations, keyed by config.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "bloom.cuh"
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

struct BloomKernels {
  uint32_t word_bytes, w, s, z, k;
  probe_fn probe;
  build_fn build;
  occ_fn probe_blocks_per_sm;
  probe_bits_fn probe_bits[kBitsVariants];
  occ_fn bits_blocks_per_sm[kBitsVariants];
  pairs_fn probe_pairs[kBitsVariants];
  occ_fn pairs_blocks_per_sm[kBitsVariants];
};

struct CuckooKernels {
  uint32_t t, b;
  probe_fn probe;
  occ_fn probe_blocks_per_sm;
  probe_bits_fn probe_bits[kBitsVariants];
  occ_fn bits_blocks_per_sm[kBitsVariants];
  void (*unpack)(const uint32_t* table, uint32_t* slots, uint32_t buckets, int grid, cudaStream_t);
  void (*insert)(const CuckooBuildArgs&, int grid, cudaStream_t);
  void (*pack)(uint32_t* table, const uint32_t* slots, uint32_t buckets, uint64_t words, int grid,
               cudaStream_t);
  void (*count)(const uint32_t* table, uint32_t buckets, uint64_t victim_word, unsigned long long* out,
                int grid, cudaStream_t);
};

void register_bloom(const BloomKernels& k);
void register_cuckoo(const CuckooKernels& k);
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
};

template <class Ops, int MINB>
struct PairsLaunch {
  static cudaError_t run(const PairsArgs& a, int grid, cudaStream_t s) {
    probe_pairs_kernel<Ops, MINB><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
  }
  static int occupancy() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, probe_pairs_kernel<Ops, MINB>, 256, 0);
    return n;
  }
};

template <class Cfg>
struct BloomLaunch {
  static cudaError_t probe(const ProbeArgs& a, int grid, cudaStream_t s) {
    probe_kernel<BloomOps<Cfg>, kProbeRounds><<<grid, kProbeThreads, 0, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t build(const BuildArgs& a, int grid, cudaStream_t s) {
    bloom_build_kernel<Cfg><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
  }
  static int occupancy() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, probe_kernel<BloomOps<Cfg>, kProbeRounds>,
                                                  kProbeThreads, 0);
    return n;
  }
};

template <typename Word, int W, int S, int Z, int K>
BloomKernels bloom_entry() {
  using C = BloomCfg<Word, W, S, Z, K>;
  using B8 = BitsLaunch<BloomOps<C>, 8>;
  using B4 = BitsLaunch<BloomOps<C>, 4>;
  using P8 = PairsLaunch<BloomOps<C>, 8>;
  using P4 = PairsLaunch<BloomOps<C>, 4>;
  return BloomKernels{static_cast<uint32_t>(sizeof(Word)), W, S, Z, K, &BloomLaunch<C>::probe,
                      &BloomLaunch<C>::build, &BloomLaunch<C>::occupancy,
                      {&B8::run, &B4::run}, {&B8::occupancy, &B4::occupancy},
                      {&P8::run, &P4::run}, {&P8::occupancy, &P4::occupancy}};
}

template <int T, int B>
struct CuckooLaunch {
  using C = CuckooCfg<T, B>;
  static cudaError_t probe(const ProbeArgs& a, int grid, cudaStream_t s) {
    probe_kernel<CuckooOps<C>, kProbeRounds><<<grid, kProbeThreads, 0, s>>>(a);
    return cudaGetLastError();
  }
  static int occupancy() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, probe_kernel<CuckooOps<C>, kProbeRounds>,
                                                  kProbeThreads, 0);
    return n;
  }
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

template <int T, int B>
CuckooKernels cuckoo_entry() {
  using L = CuckooLaunch<T, B>;
  using B8 = BitsLaunch<CuckooOps<CuckooCfg<T, B>>, 8>;
  using B4 = BitsLaunch<CuckooOps<CuckooCfg<T, B>>, 4>;
  return CuckooKernels{T, B, &L::probe, &L::occupancy, {&B8::run, &B4::run}, {&B8::occupancy, &B4::occupancy},
                       &L::unpack, &L::insert, &L::pack, &L::count};
}
#endif

}  // namespace dtlg
