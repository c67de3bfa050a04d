// probe3.cuh -- partitioned probe for filters much larger than L2.
//
// Random probes into a filter of hundreds of MiB miss L2 on most keys, fetch a
// 128-byte line per 64-byte block, and exceed the GPU's address-translation
// reach.  The partitioned probe (the radix-partitioning technique of database
// joins) first groups the probe keys by the filter range their block lies in,
// with ranges of 2^range_log2 blocks sized to sit in L2, then probes the groups
// in range order, so the filter is read from DRAM about once per pass instead
// of once per key:
//
//   1. part_hist_kernel     per-tile key count of every range
//   2. part_scan_kernel     per range: exclusive scan of the tile counts
//   3. part_scatter_kernel  (key, position) pairs into their range's segment
//   4. probe_pairs_kernel   probe each pair, set bit `position` of the
//                           key-ordered match mask (zeroed beforehand)
//   5. compact_kernel       (probe2.cuh) ascending positions from the mask
//
// Extra traffic against a direct probe: keys read twice (8 B), pairs written
// and read (16 B), all sequential.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "probe.cuh"

namespace dtlg {

constexpr int kPartThreads = 256;
constexpr int kPartKeysPerThread = 16;                  // 4 key vectors
constexpr uint32_t kPartTile = kPartThreads * kPartKeysPerThread;  // 4096 keys
constexpr int kMaxRanges = 64;

struct PartArgs {
  const uint32_t* keys_al;  // 16-byte aligned key base (see ProbeArgs)
  uint64_t n_phys;
  uint32_t pre;
  Addr addr;
  uint32_t range_log2;      // a range is 2^range_log2 consecutive blocks
  uint32_t n_ranges;
  uint32_t n_tiles;
  uint32_t* counts;         // [n_ranges][n_tiles]: counts, then exclusive prefixes
  uint32_t* totals;         // [n_ranges]
  uint2* pairs;             // (key, logical position), grouped by range
  uint32_t block_mul;       // the family constant of the block hash (C[0]; C[1]: blocked cuckoo)
};

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t key_range(uint32_t key, const PartArgs& a) {
  return block_index(key * a.block_mul, a.addr) >> a.range_log2;
}

static __global__ void __launch_bounds__(kPartThreads) part_hist_kernel(const __grid_constant__ PartArgs a) {
  __shared__ uint32_t hist[kMaxRanges];
  const uint4* keys4 = reinterpret_cast<const uint4*>(a.keys_al);
  for (uint32_t tile = blockIdx.x; tile < a.n_tiles; tile += gridDim.x) {
    for (uint32_t r = threadIdx.x; r < a.n_ranges; r += blockDim.x) hist[r] = 0;
    __syncthreads();
    const uint64_t v0 = static_cast<uint64_t>(tile) * (kPartTile / 4);
#pragma unroll
    for (int i = 0; i < kPartKeysPerThread / 4; i++) {
      const uint64_t v = v0 + static_cast<uint64_t>(i) * kPartThreads + threadIdx.x;
      const uint64_t p0 = v * 4;
      if (p0 >= a.n_phys) continue;
      const uint4 kv = __ldcs(keys4 + v);
      const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (p0 + q >= a.pre && p0 + q < a.n_phys) atomicAdd(&hist[key_range(k[q], a)], 1u);
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < a.n_ranges; r += blockDim.x)
      a.counts[static_cast<uint64_t>(r) * a.n_tiles + tile] = hist[r];
    __syncthreads();
  }
}

// One CTA per range: exclusive scan of that range's tile counts.
static __global__ void __launch_bounds__(1024) part_scan_kernel(const __grid_constant__ PartArgs a) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  const uint32_t r = blockIdx.x;
  uint32_t* c = a.counts + static_cast<uint64_t>(r) * a.n_tiles;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < a.n_tiles; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < a.n_tiles ? c[i] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= static_cast<uint32_t>(d)) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint32_t wv = s_warp[lane];
      uint32_t wi = wv;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, wi, d);
        if (lane >= static_cast<uint32_t>(d)) wi += t;
      }
      s_warp[lane] = wi - wv;
    }
    __syncthreads();
    const uint32_t carry = s_carry;
    if (i < a.n_tiles) c[i] = carry + s_warp[warp] + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = carry + s_warp[warp] + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) a.totals[r] = s_carry;
}

// Each tile is sorted by range in shared memory first, then every range's run
// is written to its segment with consecutive addresses (coalesced stores).
static __global__ void __launch_bounds__(kPartThreads) part_scatter_kernel(const __grid_constant__ PartArgs a) {
  __shared__ uint2 s_pairs[kPartTile];
  __shared__ unsigned char s_range[kPartTile];
  __shared__ uint32_t s_lbase[kMaxRanges];  // tile-local start of each range's run
  __shared__ uint32_t s_lcur[kMaxRanges];
  __shared__ uint32_t s_gbase[kMaxRanges];  // global start of this tile's part of the range
  __shared__ uint32_t s_valid;
  const uint4* keys4 = reinterpret_cast<const uint4*>(a.keys_al);
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t tile = blockIdx.x; tile < a.n_tiles; tile += gridDim.x) {
    if (threadIdx.x < 32) {
      // this tile's count per range (difference of the scanned prefixes) and
      // their exclusive scan; two ranges per lane
      uint32_t cnt[2], gb[2];
      uint32_t range_base = 0, sum_before = 0;
      for (int h = 0; h < 2; h++) {
        const uint32_t r = threadIdx.x * 2 + h;
        cnt[h] = 0;
        gb[h] = 0;
        if (r < a.n_ranges) {
          const uint32_t* c = a.counts + static_cast<uint64_t>(r) * a.n_tiles;
          const uint32_t next = tile + 1 < a.n_tiles ? c[tile + 1] : a.totals[r];
          cnt[h] = next - c[tile];
          gb[h] = c[tile];
        }
      }
      // range bases (exclusive scan of the totals) and tile-local bases
      uint32_t t0 = (threadIdx.x * 2 < a.n_ranges) ? a.totals[threadIdx.x * 2] : 0u;
      uint32_t t1 = (threadIdx.x * 2 + 1 < a.n_ranges) ? a.totals[threadIdx.x * 2 + 1] : 0u;
      uint32_t pair_tot = t0 + t1, incl = pair_tot;
      uint32_t pair_cnt = cnt[0] + cnt[1], cincl = pair_cnt;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, d);
        const uint32_t y = __shfl_up_sync(0xffffffffu, cincl, d);
        if (lane >= static_cast<uint32_t>(d)) {
          incl += x;
          cincl += y;
        }
      }
      range_base = incl - pair_tot;
      sum_before = cincl - pair_cnt;
      for (int h = 0; h < 2; h++) {
        const uint32_t r = threadIdx.x * 2 + h;
        if (r < kMaxRanges) {
          s_gbase[r] = range_base + (h ? t0 : 0u) + gb[h];
          s_lbase[r] = sum_before + (h ? cnt[0] : 0u);
          s_lcur[r] = s_lbase[r];
        }
      }
      if (threadIdx.x == 31) s_valid = cincl;
    }
    __syncthreads();
    const uint64_t v0 = static_cast<uint64_t>(tile) * (kPartTile / 4);
#pragma unroll
    for (int i = 0; i < kPartKeysPerThread / 4; i++) {
      const uint64_t v = v0 + static_cast<uint64_t>(i) * kPartThreads + threadIdx.x;
      const uint64_t p0 = v * 4;
      uint4 kv = make_uint4(0, 0, 0, 0);
      if (p0 < a.n_phys) kv = __ldcs(keys4 + v);
      const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint64_t p = p0 + q;
        const bool valid = p >= a.pre && p < a.n_phys;
        if (valid) {
          const uint32_t r = key_range(k[q], a);
          const uint32_t slot = atomicAdd(&s_lcur[r], 1u);
          s_pairs[slot] = make_uint2(k[q], static_cast<uint32_t>(p - a.pre));
          s_range[slot] = static_cast<unsigned char>(r);
        }
      }
    }
    __syncthreads();
    const uint32_t nv = s_valid;
    for (uint32_t sl = threadIdx.x; sl < nv; sl += blockDim.x) {
      const uint2 pr = s_pairs[sl];
      const uint32_t r = s_range[sl];
      __stcs(a.pairs + s_gbase[r] + (sl - s_lbase[r]), pr);
    }
    __syncthreads();
  }
}

struct PairsArgs {
  ProbeArgs probe;          // filter + addressing (keys fields unused)
  const uint2* pairs;
  uint64_t n_pairs;
  uint32_t* bits;           // key-ordered match mask (bit = physical key index), zeroed
  uint32_t pre;             // physical index of the first key
};

// Probes the pairs in range order; each match sets one bit of the mask.
template <class Ops, int MINB>
__global__ void __launch_bounds__(256, MINB) probe_pairs_kernel(const __grid_constant__ PairsArgs a) {
  const uint4* p4 = reinterpret_cast<const uint4*>(a.pairs);
  const uint64_t n2 = (a.n_pairs + 1) >> 1;  // two pairs per 16-byte vector
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n2; i += stride) {
    const uint4 x = __ldcs(p4 + i);
    const bool has2 = 2 * i + 1 < a.n_pairs;
    const bool m0 = Ops::contains(a.probe, x.x);
    const bool m1 = has2 && Ops::contains(a.probe, x.z);
    if (m0) {
      const uint64_t b = static_cast<uint64_t>(x.y) + a.pre;
      atomicOr(a.bits + (b >> 5), 1u << (b & 31u));
    }
    if (m1) {
      const uint64_t b = static_cast<uint64_t>(x.w) + a.pre;
      atomicOr(a.bits + (b >> 5), 1u << (b & 31u));
    }
  }
}

#endif  // __CUDACC__

}  // namespace dtlg
