// batched.cuh -- build and probe many filters in ONE persistent kernel.
//
// A query plan with one filter per partition or semi-join has hundreds of
// filters of very uneven size; launching a build and a probe per filter spends
// most of the time on launch latency and tail effects.  Here all filters are
// described by a table, and one persistent kernel works through a queue of three kinds of items:
//
//   build tiles:   4096 build keys of one filter;
//   range items:   one block range of a staged filter;
//   probe tiles:   4096 probe keys of one filter, tested into the filter's
//                  key-ordered match bitmask (128 words, no barrier between
//                  the warps, no look-back);
//   compact tiles: 65536 keys of one filter: ordered compaction of its
//                  bitmask into ascending match positions (per-filter
//                  decoupled look-back, as compact_kernel in probe2.cuh).
//
// The items form one queue: all build tiles, then all range items, then all
// probe tiles, then all compact tiles, each kind in filter order.  (Probing
// into a bitmask and compacting separately, as the single-filter plan 2 does,
// is 2.2x the rate of a fused probe-and-compact tile on B200: u64 w=8 s=8 k=8,
// 2^22 keys, 2^28 probes, 183 vs 83 Gkeys/s.)
//
// A build tile either inserts its keys with global atomic ORs (direct
// filters), or -- for a staged filter -- only sorts them into per-range
// buckets: the filter is cut into ranges of kBatchRangeBytes, each key goes to
// the bucket of its block's range.  A range item then builds its range in
// shared memory from its bucket (shared-memory atomics) and ORs the result
// into the filter words with coalesced read-modify-writes.  Global atomics
// are bounded by the L2's atomic throughput (about 185 G word updates/s on
// B200, so 8 per key cap a sectorized k=8 build near 23 G keys/s); staging
// turns them into streaming traffic.  A bucket that fills up sends the rest
// of its keys down the direct path, so any key distribution is built exactly.
//
// CTAs take items in queue order.  A range item of filter f waits until all
// of f's build tiles are done; a probe tile of f waits until f is built (all
// its ranges, or all its build tiles when direct).  Every item waits only on
// items earlier in the queue, which running CTAs have already taken and which
// themselves wait only on earlier items; so the bounded waits cannot deadlock.  The per-filter look-back of the ordered
// compaction is the one of probe.cuh.  Filter words are read with coherent
// loads, because they were written earlier in the same kernel.
#pragma once

#include <cstdint>
#include <type_traits>

#include "bloom.cuh"
#include "probe.cuh"

namespace dtlg {

constexpr uint32_t kBatchTile = 4096;  // keys per build or probe tile
constexpr int kBatchThreads = 256;
constexpr uint32_t kBatchRangeBytes = 32768;  // filter bytes built per range item (dynamic shared memory)
constexpr uint32_t kBatchMaxRanges = 2048;    // staged filters: at most 64 MiB

struct BatchDesc {
  Addr addr;
  uint32_t cfg;                 // index into the kernel's config menu
  void* words;
  const uint32_t* build_keys;   // 16-byte aligned
  const uint32_t* probe_keys;   // 16-byte aligned
  uint32_t* out;
  unsigned long long* count_out;
  uint32_t n_build, n_probe, match_offset;
  uint32_t n_build_tiles;               // build tiles of this filter
  uint32_t probe_tile0, n_probe_tiles;  // first global probe tile, tile count
  uint32_t ctile0, n_ctiles;            // first global compact tile (look-back word), tile count
  uint32_t* mask;                       // match bitmask, one bit per probe key (whole 128-word tiles)
  // staged build (staged != 0): range r holds blocks [r << range_shift, ...)
  uint32_t staged, n_ranges, range_shift, bucket_cap;
  uint32_t* bucket;             // n_ranges x bucket_cap keys
  unsigned int* cursor;         // per range: keys sorted in so far (zeroed)
};

// Work items of the single queue: x = kind << 30 | filter, y = the kind's index.
constexpr uint32_t kItemBuild = 0;   // y: the filter's build tile
constexpr uint32_t kItemRange = 1;   // y: the range of a staged filter
constexpr uint32_t kItemProbe = 2;   // y: the global probe tile
constexpr uint32_t kItemCompact = 3; // y: the global compact tile (look-back word)
// Probe keys a thread tests together (BloomOps::testn): their first
// loads are all in flight before any is tested.  512-filter mix, probe phase:
// 7.15 ms one at a time, 6.62 ms by two; four spill at the 64-register bound.
constexpr int kTestN = 2;
constexpr uint32_t kBatchCompactKeys = 65536;  // keys per compact tile: 8 warps x 8 rows x 32 words

struct BatchArgs {
  const BatchDesc* desc;
  uint32_t n_filters;
  const uint2* items;           // the queue, in hand-out order
  uint32_t n_items;
  unsigned long long* status;   // one look-back word per global compact tile (zeroed)
  unsigned int* probed;         // per filter: probe tiles done (zeroed)
  unsigned int* built;          // per filter: build tiles done (zeroed)
  unsigned int* ranges_built;   // per filter: range items done (zeroed)
  unsigned int* ctl;            // [0] queue head, [2] error word (zeroed)
};

#ifdef __CUDACC__

template <class Cfg0, class... Rest, class F>
__device__ __forceinline__ void dispatch_cfg(uint32_t id, F&& f) {
  if (id == 0) {
    f(Cfg0{});
  } else if constexpr (sizeof...(Rest) > 0) {
    dispatch_cfg<Rest...>(id - 1, f);
  }
}

// f(std::bool_constant<MAGIC>) for the filter's addressing mode: the block
// index is then computed without a run-time branch on it.
template <class F>
__device__ __forceinline__ void dispatch_addr(const Addr& a, F&& f) {
  if (a.magic_mode) {
    f(std::true_type{});
  } else {
    f(std::false_type{});
  }
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// Thread 0 waits (bounded) until *ctr >= need; the CTA then proceeds.  A wait
// that spins `limit` times sets bit 1 of *err and gives up.
__device__ __forceinline__ void wait_counter(const unsigned int* ctr, uint32_t need, unsigned int* err,
                                             uint32_t limit = kSpinLimit) {
  if (threadIdx.x == 0) {
    uint32_t spins = 0;
    while (ld_acquire_u32(ctr) < need) {
      if (++spins > limit) {
        atomicOr(err, 2u);
        break;
      }
      __nanosleep(128);
    }
  }
  __syncthreads();
}

// Block-wide exclusive scan of v[0..n) in place (n <= kBatchMaxRanges, 8
// entries per thread); returns the total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t* v, uint32_t n, uint32_t* s_warp) {
  constexpr uint32_t kPer = kBatchMaxRanges / kBatchThreads;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t i0 = threadIdx.x * kPer;
  uint32_t x[kPer], sum = 0;
#pragma unroll
  for (uint32_t j = 0; j < kPer; j++) {
    x[j] = i0 + j < n ? v[i0 + j] : 0u;
    sum += x[j];
  }
  uint32_t incl = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= static_cast<uint32_t>(d)) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  uint32_t before = 0, total = 0;
#pragma unroll
  for (uint32_t w = 0; w < kBatchThreads / 32; w++) {
    const uint32_t t = s_warp[w];
    before += w < warp ? t : 0u;
    total += t;
  }
  uint32_t run = before + incl - sum;
#pragma unroll
  for (uint32_t j = 0; j < kPer; j++) {
    if (i0 + j < n) v[i0 + j] = run;
    run += x[j];
  }
  __syncthreads();
  return total;
}

// Sorts one build tile of a staged filter into its range buckets.  The tile
// is first ordered by range in shared memory, so that each range's run of
// keys goes to its bucket as consecutive (coalesced) stores; one atomic per
// (tile, range) reserves the run's place in the bucket.
//   smem: s_cnt / s_gbase [kBatchMaxRanges] + s_keys [kBatchTile] = 32 KiB.
template <class Cfg, bool MAGIC>
__device__ __forceinline__ void scatter_tile(const BatchDesc& d, uint64_t k0, unsigned char* smem,
                                             uint32_t* s_warp) {
  constexpr int kRounds = kBatchTile / (kBatchThreads * 4);
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem);       // counts, then tile-local run starts
  uint32_t* s_gbase = s_cnt + kBatchMaxRanges;                // bucket position of each run
  uint32_t* s_keys = s_gbase + kBatchMaxRanges;               // the tile ordered by range
  for (uint32_t i = threadIdx.x; i < d.n_ranges; i += kBatchThreads) s_cnt[i] = 0u;
  __syncthreads();
  const uint4* k4 = reinterpret_cast<const uint4*>(d.build_keys + k0);
  uint32_t key[kRounds * 4], slot[kRounds * 4];  // slot: range << 12 | rank within the tile's run
#pragma unroll
  for (int r = 0; r < kRounds; r++) {
    const uint64_t i0 = static_cast<uint64_t>(r) * (kBatchThreads * 4) + threadIdx.x * 4u;
    uint4 kv = make_uint4(0u, 0u, 0u, 0u);
    if (k0 + i0 < d.n_build) kv = __ldcs(k4 + (i0 >> 2));
    const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      key[r * 4 + q] = k[q];
      slot[r * 4 + q] = 0xffffffffu;
      if (k0 + i0 + q < d.n_build) {
        const uint32_t rg = block_index_of<MAGIC>(k[q] * mul_const(0), d.addr) >> d.range_shift;
        slot[r * 4 + q] = (rg << 12) | atomicAdd(&s_cnt[rg], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < d.n_ranges; i += kBatchThreads) {
    const uint32_t h = s_cnt[i];
    s_gbase[i] = h ? atomicAdd(&d.cursor[i], h) : 0u;
  }
  __syncthreads();
  const uint32_t n_valid = block_exclusive_scan(s_cnt, d.n_ranges, s_warp);
#pragma unroll
  for (int j = 0; j < kRounds * 4; j++)
    if (slot[j] != 0xffffffffu) s_keys[s_cnt[slot[j] >> 12] + (slot[j] & 0xfffu)] = key[j];
  __syncthreads();
  for (uint32_t sl = threadIdx.x; sl < n_valid; sl += kBatchThreads) {
    const uint32_t kk = s_keys[sl];
    const uint32_t rg = block_index_of<MAGIC>(kk * mul_const(0), d.addr) >> d.range_shift;
    const uint32_t pos = s_gbase[rg] + (sl - s_cnt[rg]);
    if (pos < d.bucket_cap) {
      d.bucket[static_cast<uint64_t>(rg) * d.bucket_cap + pos] = kk;
    } else {
      BloomOps<Cfg>::insert(d.words, kk, d.addr);  // bucket full: direct path
    }
  }
}

// Builds range rg of a staged filter in shared memory and ORs it into the words.
template <class Cfg, bool MAGIC>
__device__ __forceinline__ void build_range(const BatchDesc& d, uint32_t rg, unsigned char* smem) {
  using Word = typename Cfg::word_t;
  constexpr uint32_t kW = Cfg::kW;
  Word* s_w = reinterpret_cast<Word*>(smem);
  const uint32_t blk0 = rg << d.range_shift;
  const uint32_t nblk = min(1u << d.range_shift, d.addr.block_cnt - blk0);
  const uint32_t nw = nblk * kW;
  for (uint32_t i = threadIdx.x; i < nw; i += kBatchThreads) s_w[i] = 0;
  __syncthreads();
  const uint32_t cnt = min(ld_weak_32(d.cursor + rg), d.bucket_cap);
  const uint32_t* bk = d.bucket + static_cast<uint64_t>(rg) * d.bucket_cap;
  // The range's words sit in shared memory with the word index of local block
  // b XORed with bits 1.. of b: a 64-byte block spans 16 of the 32 banks, so
  // word w of random blocks would fall on just 2 (u32 words) or 4 (u64 halves)
  // banks, and a warp's atomics on the same word of 32 blocks would conflict
  // 8 to 16 ways; swizzled they spread over 16 or 32 banks.
  // kU bucket keys per thread in flight: each load comes from L2 or DRAM, and
  // one at a time left the loop waiting on it (long scoreboard)
  constexpr int kU = 4;
  for (uint32_t i0 = 0; i0 < cnt; i0 += kBatchThreads * kU) {
    uint32_t kk[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const uint32_t i = i0 + u * kBatchThreads + threadIdx.x;
      kk[u] = i < cnt ? ld_weak_32(bk + i) : 0u;
    }
#pragma unroll
    for (int u = 0; u < kU; u++) {
      if (i0 + u * kBatchThreads + threadIdx.x >= cnt) break;
      const uint32_t key = kk[u];
      const uint32_t lb = block_index_of<MAGIC>(key * mul_const(0), d.addr) - blk0;
      const uint32_t swz = (lb >> 1) & (kW - 1);
      Word* base = s_w + static_cast<uint64_t>(lb) * kW;
      static_for<BloomOps<Cfg>::kS.ng>([&](auto G) {
        constexpr int g = decltype(G)::value;
        Word* p = base + (BloomOps<Cfg>::template group_word<g>(key) ^ swz);
        constexpr Group grp = BloomOps<Cfg>::kS.g[g];
        if constexpr (sizeof(Word) == 8 && grp.nbit == 1) {
          // one bit: one 32-bit atomic on the half that holds it, no test
          constexpr BitDraw b = grp.bit[0];
          const uint32_t bit = ((hash_sel<b.sel>(key) >> b.shift) & ((1u << b.bits) - 1u)) + b.off;
          atomicOr(reinterpret_cast<uint32_t*>(p) + (bit >> 5), 1u << (bit & 31u));
          return;
        }
        const Word m = BloomOps<Cfg>::template group_mask<g>(key);
        if constexpr (sizeof(Word) == 8) {
          // 32-bit shared-memory atomics on the halves that have bits to set
          uint32_t* p32 = reinterpret_cast<uint32_t*>(p);
          const uint32_t lo = static_cast<uint32_t>(m), hi = static_cast<uint32_t>(m >> 32);
          if (lo) atomicOr(p32, lo);
          if (hi) atomicOr(p32 + 1, hi);
        } else {
          atomicOr(reinterpret_cast<uint32_t*>(p), static_cast<uint32_t>(m));
        }
      });
    }
  }
  __syncthreads();
  Word* gw = static_cast<Word*>(d.words) + static_cast<uint64_t>(blk0) * kW;
  for (uint32_t i0 = 0; i0 < nw; i0 += kBatchThreads * kU) {
    Word v[kU], w[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const uint32_t i = i0 + u * kBatchThreads + threadIdx.x;
      v[u] = i < nw ? s_w[i ^ ((i / kW >> 1) & (kW - 1))] : Word(0);  // word i % kW of block i / kW, unswizzled
      w[u] = 0;
      if (v[u] != 0) {
        if constexpr (sizeof(Word) == 8) {
          w[u] = static_cast<Word>(ld_weak_64(gw + i));
        } else {
          w[u] = static_cast<Word>(ld_weak_32(gw + i));
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kU; u++) {
      if (v[u] != 0) gw[i0 + u * kBatchThreads + threadIdx.x] = w[u] | v[u];
    }
  }
}

// Four CTAs per SM: -Xptxas -v gives 64 registers and no spills with this
// bound, where ptxas left to itself also chose 64 registers but spilled
// (68 bytes of stores, 56 of loads per thread).
template <class... Cfgs>
__global__ void __launch_bounds__(kBatchThreads, 4) batched_kernel(const __grid_constant__ BatchArgs a) {
  constexpr int kRounds = kBatchTile / (kBatchThreads * 4);  // 4 rounds of 1024 keys
  constexpr int kWarps = kBatchThreads / 32;
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_wtot[kRounds * kWarps];
  __shared__ uint32_t s_excl;
  extern __shared__ __align__(16) unsigned char s_dyn[];  // kBatchRangeBytes
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;

  // filters without probe keys report a zero count
  if (blockIdx.x == 0) {
    for (uint32_t f = threadIdx.x; f < a.n_filters; f += blockDim.x)
      if (a.desc[f].n_probe == 0) *a.desc[f].count_out = 0ull;
  }

  ProbeArgs lb{};  // look-back state: status words + error word
  lb.status = a.status;
  lb.err = &a.ctl[2];
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&a.ctl[0], 1u);
    __syncthreads();
    const uint32_t item = s_tile;
    __syncthreads();
    if (item >= a.n_items) break;
    const uint2 it = a.items[item];
    const uint32_t kind = it.x >> 30, f = it.x & 0x3fffffffu;
    const BatchDesc& d = a.desc[f];

    if (kind == kItemBuild) {
      const uint64_t k0 = static_cast<uint64_t>(it.y) * kBatchTile;
      dispatch_cfg<Cfgs...>(d.cfg, [&](auto c) {
        using Cfg = decltype(c);
        if (d.staged) {
          dispatch_addr(d.addr, [&](auto m) { scatter_tile<Cfg, decltype(m)::value>(d, k0, s_dyn, s_wtot); });
          return;
        }
        using Ops = BloomOps<Cfg>;
        const uint4* k4 = reinterpret_cast<const uint4*>(d.build_keys + k0);
        if constexpr (Ops::kLaneInsert && sizeof(typename Ops::LaneStage) * (kBatchThreads / 32) <= kBatchRangeBytes) {
          // warp-cooperative inserts (BloomOps::insert_lanes), staged in s_dyn
          typename Ops::LaneStage& my = reinterpret_cast<typename Ops::LaneStage*>(s_dyn)[threadIdx.x >> 5];
#pragma unroll
          for (int r = 0; r < kRounds; r++) {
            const uint64_t i0 = static_cast<uint64_t>(r) * (kBatchThreads * 4) + threadIdx.x * 4u;
            const uint4 kv = k0 + i0 < d.n_build ? __ldcs(k4 + (i0 >> 2)) : make_uint4(0, 0, 0, 0);
            const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
            for (int q = 0; q < 4; q++) Ops::insert_lanes(d.words, k[q], k0 + i0 + q < d.n_build, d.addr, my);
          }
        } else {
#pragma unroll
          for (int r = 0; r < kRounds; r++) {
            const uint64_t i0 = static_cast<uint64_t>(r) * (kBatchThreads * 4) + threadIdx.x * 4u;
            if (k0 + i0 >= d.n_build) continue;
            const uint4 kv = __ldcs(k4 + (i0 >> 2));
            const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
            for (int q = 0; q < 4; q++)
              if (k0 + i0 + q < d.n_build) Ops::insert(d.words, k[q], d.addr);
          }
        }
      });
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&a.built[f], 1u);
      }
      continue;
    }

    if (kind == kItemRange) {
      wait_counter(&a.built[f], d.n_build_tiles, &a.ctl[2]);
      dispatch_cfg<Cfgs...>(d.cfg, [&](auto c) {
        dispatch_addr(d.addr, [&](auto m) { build_range<decltype(c), decltype(m)::value>(d, it.y, s_dyn); });
      });
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&a.ranges_built[f], 1u);
      }
      continue;
    }

    if (kind == kItemProbe) {
      const uint32_t tile = it.y;
      const uint32_t local = tile - d.probe_tile0;
      if (d.staged) {
        wait_counter(&a.ranges_built[f], d.n_ranges, &a.ctl[2]);
      } else {
        wait_counter(&a.built[f], d.n_build_tiles, &a.ctl[2]);
      }
      const uint64_t k0 = static_cast<uint64_t>(local) * kBatchTile;
      const uint32_t n_words = (d.n_probe + 31u) / 32u;
      // blocks of >= 32 bytes are read with 256-bit loads when the words are 32-byte aligned
      const bool vec32 = (reinterpret_cast<uintptr_t>(d.words) & 31u) == 0;
      dispatch_cfg<Cfgs...>(d.cfg, [&](auto c) { dispatch_addr(d.addr, [&](auto m) {
        using Cfg = decltype(c);
        constexpr bool MAGIC = decltype(m)::value;
        const uint4* k4 = reinterpret_cast<const uint4*>(d.probe_keys + k0);
#pragma unroll 2
        for (int r = 0; r < kRounds; r++) {
          const uint32_t i0 = r * (kBatchThreads * 4) + threadIdx.x * 4u;
          uint32_t fl = 0;
          if (k0 + i0 < d.n_probe) {
            const uint4 kv = __ldcs(k4 + (i0 >> 2));
            const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
            const typename Cfg::word_t* base[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
              const uint32_t blk = block_index_of<MAGIC>(k[q] * mul_const(0), d.addr);
              base[q] = static_cast<const typename Cfg::word_t*>(d.words) + static_cast<uint64_t>(blk) * Cfg::kW;
            }
            uint32_t hit = 0;
#pragma unroll
            for (int g0 = 0; g0 < 4; g0 += kTestN)
              hit |= BloomOps<Cfg>::template testn<kTestN, false>(base + g0, k + g0, (1u << kTestN) - 1u, vec32) << g0;
#pragma unroll
            for (int q = 0; q < 4; q++) fl |= ((((hit >> q) & 1u) && k0 + i0 + q < d.n_probe) ? 1u : 0u) << q;
          }
          // lanes 8j .. 8j+7 hold keys 32j .. 32j+31 of the warp's 128: word j
          uint32_t x = fl << (4u * (lane & 7u));
          x |= __shfl_xor_sync(0xffffffffu, x, 1);
          x |= __shfl_xor_sync(0xffffffffu, x, 2);
          x |= __shfl_xor_sync(0xffffffffu, x, 4);
          const uint32_t w = local * (kBatchTile / 32) + r * (kBatchThreads * 4 / 32) + warp * 4 + (lane >> 3);
          if ((lane & 7u) == 0 && w < n_words) __stcg(d.mask + w, x);
        }
      }); });
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&a.probed[f], 1u);
      }
      continue;
    }

    // kItemCompact: ordered compaction of 65536 keys' match bits.  Warp w owns
    // the 256 words w*256 .. w*256+255 of the tile as 8 rows of 32 (lane l
    // holds word row*32 + l); the tile's offset comes from the look-back over
    // this filter's compact tiles, the warp's from a CTA scan, a row's from a
    // warp scan; a row's matches are staged in shared memory in key order and
    // stored by the whole warp to consecutive slots.
    const uint32_t ct = it.y;
    const uint32_t local = ct - d.ctile0;
    wait_counter(&a.probed[f], d.n_probe_tiles, &a.ctl[2]);
    constexpr int kRows = 8;
    const uint32_t n_words = (d.n_probe + 31u) / 32u;
    const uint64_t wbase = static_cast<uint64_t>(local) * (kBatchCompactKeys / 32) + warp * (kRows * 32);
    uint32_t wv[kRows];
    uint32_t cnt = 0;
#pragma unroll
    for (int i = 0; i < kRows; i++) {
      const uint64_t idx = wbase + static_cast<uint64_t>(i) * 32 + lane;
      wv[i] = idx < n_words ? __ldcg(d.mask + idx) : 0u;
      cnt += __popc(wv[i]);
    }
#pragma unroll
    for (int dd = 16; dd > 0; dd >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, dd);
    if (lane == 0) s_wtot[warp] = cnt;
    __syncthreads();
    if (warp == 0) {
      const uint32_t v = lane < kWarps ? s_wtot[lane] : 0u;
      uint32_t wi = v;
#pragma unroll
      for (int dd = 1; dd < kWarps; dd <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, wi, dd);
        if (lane >= static_cast<uint32_t>(dd)) wi += t;
      }
      const uint32_t agg = __shfl_sync(0xffffffffu, wi, kWarps - 1);
      if (lane < kWarps) s_wtot[lane] = wi - v;
      uint32_t excl = 0;
      if (local == 0) {
        if (lane == 0) st_volatile(a.status + ct, kFlagPrefix | agg);
      } else {
        if (lane == 0) st_volatile(a.status + ct, kFlagAgg | agg);
        // look back over this filter's earlier compact tiles only
        ProbeArgs fl = lb;
        fl.status = a.status + d.ctile0;
        excl = look_back(fl, local, lane);
        if (lane == 0) st_volatile(a.status + ct, kFlagPrefix | static_cast<uint32_t>(excl + agg));
      }
      if (lane == 0) {
        s_excl = excl;
        if (local == d.n_ctiles - 1) {
          const bool failed = *reinterpret_cast<volatile unsigned int*>(&a.ctl[2]) != 0u;
          *d.count_out = failed ? ~0ull : static_cast<unsigned long long>(excl) + agg;
        }
      }
    }
    __syncthreads();
    uint32_t pos = s_excl + s_wtot[warp];
    uint32_t* stage = reinterpret_cast<uint32_t*>(s_dyn) + warp * 1024;  // 8 x 4 KiB of the 32 KiB
#pragma unroll
    for (int i = 0; i < kRows; i++) {
      const uint32_t ci = __popc(wv[i]);
      uint32_t incl = ci;
#pragma unroll
      for (int dd = 1; dd < 32; dd <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, dd);
        if (lane >= static_cast<uint32_t>(dd)) incl += t;
      }
      const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
      if (tot == 0) continue;
      const uint32_t first = static_cast<uint32_t>((wbase + static_cast<uint64_t>(i) * 32 + lane) * 32);
      uint32_t m = wv[i];
      uint32_t o = incl - ci;
      while (m) {
        const uint32_t b = __ffs(m) - 1;
        m &= m - 1;
        stage[o++] = first + b;
      }
      __syncwarp();
      for (uint32_t j = lane; j < tot; j += 32) __stcs(d.out + pos + j, stage[j] + d.match_offset);
      __syncwarp();
      pos += tot;
    }
    __syncthreads();
  }
}

#endif  // __CUDACC__

}  // namespace dtlg
