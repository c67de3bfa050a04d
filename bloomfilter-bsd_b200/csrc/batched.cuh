// batched.cuh -- build and probe many filters in ONE persistent kernel.
//
// A query plan with one filter per partition or semi-join has hundreds of
// filters of very uneven size; launching a build and a probe per filter spends
// most of the time on launch latency and tail effects.  Here all filters are
// described by a table, and one persistent kernel works through three queues:
//
//   build queue: tiles of 4096 build keys, over all filters;
//   range queue: (filter, block range) items of staged filters;
//   probe queue: tiles of 4096 probe keys, over all filters, each filter's
//                tiles in order (per-filter ordered compaction).
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
// CTAs drain the queues in order.  A range item of filter f waits until all
// of f's build tiles are done; a probe tile of f waits until f is built (all
// its ranges, or all its build tiles when direct).  The waits are bounded and
// cannot deadlock: by the time an item of a later queue is handed out, every
// item of the earlier queues has been taken by a running CTA, and those only
// wait on queues earlier still.  The per-filter look-back of the ordered
// compaction is the one of probe.cuh.  Filter words are read with coherent
// loads, because they were written earlier in the same kernel.
#pragma once

#include <cstdint>

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
  uint32_t build_tile0, n_build_tiles;  // first global build tile, tile count
  uint32_t probe_tile0, n_probe_tiles;  // first global probe tile, tile count
  uint32_t vec32;
  // staged build (staged != 0): range r holds blocks [r << range_shift, ...)
  uint32_t staged, n_ranges, range_shift, bucket_cap;
  uint32_t* bucket;             // n_ranges x bucket_cap keys
  unsigned int* cursor;         // per range: keys sorted in so far (zeroed)
};

struct BatchArgs {
  const BatchDesc* desc;
  uint32_t n_filters;
  const uint32_t* build_map;    // global build tile -> filter
  const uint32_t* probe_map;    // global probe tile -> filter
  uint32_t n_build_tiles, n_probe_tiles;
  unsigned long long* status;   // one look-back word per global probe tile (zeroed)
  unsigned int* built;          // per filter: build tiles done (zeroed)
  unsigned int* ranges_built;   // per filter: range items done (zeroed)
  const uint2* range_items;     // range queue: (filter, range)
  uint32_t n_range_items;
  unsigned int* ctl;            // [0] build, [1] probe, [3] range queue heads, [2] error word (zeroed)
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

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// Thread 0 waits (bounded) until *ctr >= need; the CTA then proceeds.
__device__ __forceinline__ void wait_counter(const unsigned int* ctr, uint32_t need, unsigned int* err) {
  if (threadIdx.x == 0) {
    uint32_t spins = 0;
    while (ld_acquire_u32(ctr) < need) {
      if (++spins > kSpinLimit) {
        atomicOr(err, 2u);
        break;
      }
      __nanosleep(128);
    }
  }
  __syncthreads();
}

// Sorts one build tile of a staged filter into its range buckets.
template <class Cfg>
__device__ __forceinline__ void scatter_tile(const BatchDesc& d, uint64_t k0, uint32_t* s_hist, uint32_t* s_base) {
  constexpr int kRounds = kBatchTile / (kBatchThreads * 4);
  for (uint32_t i = threadIdx.x; i < d.n_ranges; i += kBatchThreads) s_hist[i] = 0u;
  __syncthreads();
  const uint4* k4 = reinterpret_cast<const uint4*>(d.build_keys + k0);
  uint32_t key[kRounds * 4], slot[kRounds * 4];  // slot: range << 12 | index within the tile's share
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
        const uint32_t rg = block_index(k[q] * mul_const(0), d.addr) >> d.range_shift;
        slot[r * 4 + q] = (rg << 12) | atomicAdd(&s_hist[rg], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < d.n_ranges; i += kBatchThreads) {
    const uint32_t h = s_hist[i];
    s_base[i] = h ? atomicAdd(&d.cursor[i], h) : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kRounds * 4; j++) {
    if (slot[j] == 0xffffffffu) continue;
    const uint32_t rg = slot[j] >> 12;
    const uint32_t pos = s_base[rg] + (slot[j] & 0xfffu);
    if (pos < d.bucket_cap) {
      d.bucket[static_cast<uint64_t>(rg) * d.bucket_cap + pos] = key[j];
    } else {
      BloomOps<Cfg>::insert(d.words, key[j], d.addr);  // bucket full: direct path
    }
  }
}

// Builds range rg of a staged filter in shared memory and ORs it into the words.
template <class Cfg>
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
  for (uint32_t i = threadIdx.x; i < cnt; i += kBatchThreads) {
    const uint32_t key = ld_weak_32(bk + i);
    Word* base = s_w + static_cast<uint64_t>(block_index(key * mul_const(0), d.addr) - blk0) * kW;
    static_for<BloomOps<Cfg>::kS.ng>([&](auto G) {
      constexpr int g = decltype(G)::value;
      Word* p = base + BloomOps<Cfg>::template group_word<g>(key);
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
  __syncthreads();
  Word* gw = static_cast<Word*>(d.words) + static_cast<uint64_t>(blk0) * kW;
  for (uint32_t i = threadIdx.x; i < nw; i += kBatchThreads) {
    const Word v = s_w[i];
    if (v == 0) continue;
    if constexpr (sizeof(Word) == 8) {
      gw[i] = static_cast<Word>(ld_weak_64(gw + i)) | v;
    } else {
      gw[i] = static_cast<Word>(ld_weak_32(gw + i)) | v;
    }
  }
}

template <class... Cfgs>
__global__ void __launch_bounds__(kBatchThreads) batched_kernel(const __grid_constant__ BatchArgs a) {
  constexpr int kRounds = kBatchTile / (kBatchThreads * 4);  // 4 rounds of 1024 keys
  constexpr int kWarps = kBatchThreads / 32;
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_wtot[kRounds * kWarps];
  __shared__ uint32_t s_excl;
  extern __shared__ __align__(16) unsigned char s_dyn[];  // kBatchRangeBytes
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;

  // filters without probe keys report a zero count
  if (blockIdx.x == 0) {
    for (uint32_t f = threadIdx.x; f < a.n_filters; f += blockDim.x)
      if (a.desc[f].n_probe == 0) *a.desc[f].count_out = 0ull;
  }

  // ---- build queue ----
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&a.ctl[0], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    __syncthreads();
    if (tile >= a.n_build_tiles) break;
    const uint32_t f = a.build_map[tile];
    const BatchDesc& d = a.desc[f];
    const uint64_t k0 = static_cast<uint64_t>(tile - d.build_tile0) * kBatchTile;
    dispatch_cfg<Cfgs...>(d.cfg, [&](auto c) {
      using Cfg = decltype(c);
      if (d.staged) {
        uint32_t* s_hist = reinterpret_cast<uint32_t*>(s_dyn);
        scatter_tile<Cfg>(d, k0, s_hist, s_hist + kBatchMaxRanges);
        return;
      }
      const uint4* k4 = reinterpret_cast<const uint4*>(d.build_keys + k0);
#pragma unroll
      for (int r = 0; r < kRounds; r++) {
        const uint64_t i0 = static_cast<uint64_t>(r) * (kBatchThreads * 4) + threadIdx.x * 4u;
        if (k0 + i0 >= d.n_build) continue;
        const uint4 kv = __ldcs(k4 + (i0 >> 2));
        const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (k0 + i0 + q < d.n_build) BloomOps<Cfg>::insert(d.words, k[q], d.addr);
      }
    });
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&a.built[f], 1u);
    }
  }

  // ---- range queue (staged filters) ----
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&a.ctl[3], 1u);
    __syncthreads();
    const uint32_t item = s_tile;
    __syncthreads();
    if (item >= a.n_range_items) break;
    const uint2 fr = a.range_items[item];
    const BatchDesc& d = a.desc[fr.x];
    wait_counter(&a.built[fr.x], d.n_build_tiles, &a.ctl[2]);
    dispatch_cfg<Cfgs...>(d.cfg, [&](auto c) { build_range<decltype(c)>(d, fr.y, s_dyn); });
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&a.ranges_built[fr.x], 1u);
    }
  }

  // ---- probe queue ----
  ProbeArgs lb{};  // look-back state: status words + error word
  lb.status = a.status;
  lb.err = &a.ctl[2];
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&a.ctl[1], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= a.n_probe_tiles) break;
    const uint32_t f = a.probe_map[tile];
    const BatchDesc& d = a.desc[f];
    const uint32_t local = tile - d.probe_tile0;
    if (d.staged) {
      wait_counter(&a.ranges_built[f], d.n_ranges, &a.ctl[2]);
    } else {
      wait_counter(&a.built[f], d.n_build_tiles, &a.ctl[2]);
    }
    const uint64_t k0 = static_cast<uint64_t>(local) * kBatchTile;
    uint32_t flags[kRounds];
    uint32_t lane_excl[kRounds];
    dispatch_cfg<Cfgs...>(d.cfg, [&](auto c) {
      using Cfg = decltype(c);
      const uint4* k4 = reinterpret_cast<const uint4*>(d.probe_keys + k0);
#pragma unroll
      for (int r = 0; r < kRounds; r++) {
        const uint64_t i0 = static_cast<uint64_t>(r) * (kBatchThreads * 4) + threadIdx.x * 4u;
        uint32_t fl = 0;
        if (k0 + i0 < d.n_probe) {
          const uint4 kv = __ldcs(k4 + (i0 >> 2));
          const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const uint32_t blk = block_index(k[q] * mul_const(0), d.addr);
            const auto* base = static_cast<const typename Cfg::word_t*>(d.words) +
                               static_cast<uint64_t>(blk) * Cfg::kW;
            const bool hit = BloomOps<Cfg>::template test_block<false>(base, k[q], false);
            fl |= ((hit && k0 + i0 + q < d.n_probe) ? 1u : 0u) << q;
          }
        }
        flags[r] = fl;
      }
    });
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      uint32_t tot = 0, ex = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint32_t b = __ballot_sync(0xffffffffu, (flags[r] >> q) & 1u);
        ex += __popc(b & lt_mask);
        tot += __popc(b);
      }
      lane_excl[r] = ex;
      if (lane == 0) s_wtot[r * kWarps + warp] = tot;
    }
    __syncthreads();
    if (warp == 0) {
      const uint32_t v = lane < kRounds * kWarps ? s_wtot[lane] : 0u;
      uint32_t incl = v;
#pragma unroll
      for (int dd = 1; dd < 32; dd <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, dd);
        if (lane >= static_cast<uint32_t>(dd)) incl += t;
      }
      const uint32_t agg = __shfl_sync(0xffffffffu, incl, 31);
      if (lane < kRounds * kWarps) s_wtot[lane] = incl - v;
      uint32_t excl = 0;
      if (local == 0) {
        if (lane == 0) st_volatile(a.status + tile, kFlagPrefix | agg);
      } else {
        if (lane == 0) st_volatile(a.status + tile, kFlagAgg | agg);
        // look back over this filter's earlier tiles only (global tiles
        // probe_tile0 .. tile-1): the helper sees a status array that
        // starts at this filter's first tile
        ProbeArgs fl = lb;
        fl.status = a.status + d.probe_tile0;
        excl = look_back(fl, local, lane);
        if (lane == 0) st_volatile(a.status + tile, kFlagPrefix | static_cast<uint32_t>(excl + agg));
      }
      if (lane == 0) {
        s_excl = excl;
        if (local == d.n_probe_tiles - 1) {
          const bool failed = *reinterpret_cast<volatile unsigned int*>(&a.ctl[2]) != 0u;
          *d.count_out = failed ? ~0ull : static_cast<unsigned long long>(excl) + agg;
        }
      }
    }
    __syncthreads();
    const uint32_t excl = s_excl;
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      uint32_t fl = flags[r];
      if (fl == 0) continue;
      uint32_t pos = excl + s_wtot[r * kWarps + warp] + lane_excl[r];
      const uint32_t i0 = static_cast<uint32_t>(k0) + r * (kBatchThreads * 4) + threadIdx.x * 4u;
      while (fl) {
        const int q = __ffs(fl) - 1;
        fl &= fl - 1;
        __stcs(d.out + pos, i0 + static_cast<uint32_t>(q) + d.match_offset);
        pos++;
      }
    }
    __syncthreads();
  }
}

#endif  // __CUDACC__

}  // namespace dtlg
