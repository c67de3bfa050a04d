// probe.cuh -- batch_contains as one pass: probe + ordered match compaction.
//
// Contract (blocked_bloomfilter_batch_dispatch.hpp:29-69, filter_base.hpp:34-45):
// write i + match_offset (32-bit wrap) for every matching key index i, in
// ascending order, and return the count.
//
// Shape: persistent CTAs of 256 threads pull tiles of 1024*ROUNDS keys from a
// device counter (so a tile is only ever taken after all earlier tiles were
// taken by running CTAs: the look-back below cannot deadlock).  Inside a tile,
// thread t of round r owns the 4 consecutive keys r*1024 + 4t .. +3, loaded as
// one 16-byte vector; matches are ranked with warp ballots and a CTA scan, and
// the tile's global offset comes from a decoupled look-back over the per-tile
// status words.  Every wait is bounded: on timeout the kernel raises the error
// word and carries on with a zero prefix, so it always terminates.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace dtlg {

struct ProbeArgs {
  const void* filter;           // Bloom words / cuckoo table (+ victim record)
  const uint32_t* keys_al;      // keys rounded down to a 16-byte boundary
  uint64_t n_phys;              // pre + key_cnt
  uint32_t pre;                 // keys_al[0 .. pre) precede the first key
  uint32_t match_offset;
  uint32_t* out;                // match positions
  unsigned long long* count_out;  // device: total match count
  unsigned long long* status;   // per-tile look-back words (zeroed)
  unsigned int* tile_ctr;       // tile queue head (zeroed)
  unsigned int* err;            // error word (zeroed); bit 0 = wait timed out
  uint32_t n_tiles;
  Addr addr;
  uint64_t victim_word;         // cuckoo: 32-bit word index of the victim record
  // Block-range pass (two-pass probe only; all zero = off): a key whose block
  // (bucket) lies outside [blk_lo, blk_hi) is not probed in this pass.
  uint32_t range_on, blk_lo, blk_hi;
  // 1 when the filter base is 32-byte aligned: blocks of >= 32 bytes are then
  // read with 256-bit loads.
  uint32_t vec32;
  // 1: a Bloom filter's 256-bit block loads do not allocate in L1 (bitmask
  // plan, filters that cannot live in L1; set by the planner)
  uint32_t l1na;
  // blocked cuckoo filter: log2(buckets per block), and the shift that turns
  // the block hash into the bucket hash (32: the bucket hash is key * C[0])
  uint32_t bcf_bucket_bits, bcf_hash_shift;
  // classic Bloom filter: bits per key, and the bit index (h >> shift) & mask
  uint32_t cbf_k, cbf_bit_shift, cbf_bit_mask;
};

constexpr int kProbeThreads = 256;
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagPrefix = 2ull << 62;
constexpr uint32_t kSpinLimit = 1u << 22;  // ~ seconds with the backoff below

#ifdef __CUDACC__

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ void st_volatile(unsigned long long* p, unsigned long long v) {
  *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

// Exclusive prefix of this tile from the predecessors' status words (warp 0).
// A wait that spins `limit` times sets bit 0 of *a.err and returns what it has.
__device__ __forceinline__ uint32_t look_back(const ProbeArgs& a, uint32_t tile, uint32_t lane,
                                              uint32_t limit = kSpinLimit) {
  uint32_t excl = 0;
  int64_t pred = static_cast<int64_t>(tile) - 1;
  uint32_t spins = 0;
  while (pred >= 0) {
    const int64_t idx = pred - static_cast<int64_t>(lane);
    const unsigned long long st = idx >= 0 ? ld_volatile(a.status + idx) : kFlagPrefix;
    const unsigned long long flag = st & (3ull << 62);
    const uint32_t not_ready = __ballot_sync(0xffffffffu, flag == 0);
    const uint32_t prefix = __ballot_sync(0xffffffffu, flag == kFlagPrefix);
    // lanes 0..fp (nearest predecessors first) must all be ready
    const uint32_t need = prefix ? ((prefix & (0u - prefix)) << 1) - 1u : 0xffffffffu;
    if (not_ready & need) {
      if (++spins > limit) {
        if (lane == 0) atomicOr(a.err, 1u);
        break;
      }
      __nanosleep(64);
      continue;
    }
    uint32_t v = (need >> lane) & 1u ? static_cast<uint32_t>(st) : 0u;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    excl += v;
    if (prefix) break;
    pred -= 32;
  }
  return excl;
}

// Ops::contains(const ProbeArgs&, uint32_t key) -> bool, branch-free and safe
// for any key value (block / bucket indexes are always inside the filter).
template <class Ops, int ROUNDS>
__global__ void __launch_bounds__(kProbeThreads)
probe_kernel(const __grid_constant__ ProbeArgs a) {
  constexpr int kTile = kProbeThreads * 4 * ROUNDS;
  constexpr int kWarps = kProbeThreads / 32;
  static_assert(ROUNDS * kWarps <= 32, "one warp scans the warp totals");
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_wtot[ROUNDS * kWarps];
  __shared__ uint32_t s_excl;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint4* keys4 = reinterpret_cast<const uint4*>(a.keys_al);

  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= a.n_tiles) break;
    const uint64_t tbase = static_cast<uint64_t>(tile) * kTile;

    uint32_t flags[ROUNDS];
    uint32_t lane_excl[ROUNDS];
#pragma unroll
    for (int r = 0; r < ROUNDS; r++) {
      const uint64_t p0 = tbase + static_cast<uint64_t>(r) * (kProbeThreads * 4) + threadIdx.x * 4u;
      uint32_t f = 0;
      if (p0 < a.n_phys) {
        const uint4 kv = __ldcs(keys4 + (p0 >> 2));
        const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
        for (int q = 0; q < 4; q++) f |= (Ops::contains(a, k[q]) ? 1u : 0u) << q;
        // drop lanes before the first key and past the last one
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const uint64_t p = p0 + q;
          if (p < a.pre || p >= a.n_phys) f &= ~(1u << q);
        }
      }
      flags[r] = f;
      uint32_t tot = 0, ex = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint32_t b = __ballot_sync(0xffffffffu, (f >> q) & 1u);
        ex += __popc(b & lt_mask);
        tot += __popc(b);
      }
      lane_excl[r] = ex;
      if (lane == 0) s_wtot[r * kWarps + warp] = tot;
    }
    __syncthreads();

    if (warp == 0) {
      // exclusive scan of the warp totals in key order (round-major)
      const uint32_t v = lane < ROUNDS * kWarps ? s_wtot[lane] : 0u;
      uint32_t incl = v;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= static_cast<uint32_t>(d)) incl += t;
      }
      const uint32_t agg = __shfl_sync(0xffffffffu, incl, 31);
      if (lane < ROUNDS * kWarps) s_wtot[lane] = incl - v;
      uint32_t excl = 0;
      if (tile == 0) {
        if (lane == 0) st_volatile(a.status, kFlagPrefix | agg);
      } else {
        if (lane == 0) st_volatile(a.status + tile, kFlagAgg | agg);
        excl = look_back(a, tile, lane);
        if (lane == 0) st_volatile(a.status + tile, kFlagPrefix | static_cast<uint32_t>(excl + agg));
      }
      if (lane == 0) {
        s_excl = excl;
        if (tile == a.n_tiles - 1) {
          const bool failed = *reinterpret_cast<volatile unsigned int*>(a.err) != 0u;
          *a.count_out = failed ? ~0ull : static_cast<unsigned long long>(excl) + agg;
        }
      }
    }
    __syncthreads();

    const uint32_t excl = s_excl;
#pragma unroll
    for (int r = 0; r < ROUNDS; r++) {
      uint32_t f = flags[r];
      if (f == 0) continue;
      uint32_t pos = excl + s_wtot[r * kWarps + warp] + lane_excl[r];
      const uint64_t p0 = tbase + static_cast<uint64_t>(r) * (kProbeThreads * 4) + threadIdx.x * 4u;
      const uint32_t logical0 = static_cast<uint32_t>(p0 - a.pre);
      while (f) {
        const int q = __ffs(f) - 1;
        f &= f - 1;
        __stcs(a.out + pos, logical0 + static_cast<uint32_t>(q) + a.match_offset);
        pos++;
      }
    }
    __syncthreads();
  }
}

#endif  // __CUDACC__

}  // namespace dtlg
