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
//   1. part_scatter_kernel    one pass over the keys: each 4096-key tile is
//                             sorted by range in shared memory, reserves room
//                             for its run of every range with one atomic add
//                             on that range's fill counter, and writes the
//                             runs as (key, position) pairs into the range's
//                             segment
//   2. probe_pairs_kernel     probe the segments chunk by chunk in range
//                             order; each match sets bit `position` of the
//                             key-ordered match mask (zeroed beforehand)
//   3. probe_overflow_kernel  the keys of runs that did not fit (see below)
//   4. compact_kernel         (probe2.cuh) ascending positions from the mask
//
// No counting pass: every segment has a fixed capacity, the range's expected
// share of the keys (its block count over the filter's) plus 1/32 and one
// tile, so the keys are read once.  For hashed keys the share is exceeded by
// far less than that slack (at 2^28 keys the slack is ~60 standard deviations).
// Whatever does not fit is still probed: the tile records, per range, that its
// run overflowed, and the overflow kernel re-probes those keys straight from
// the key array (a key probed twice sets the same mask bit twice).  Where a
// second insert of a key is not harmless (blocked cuckoo builds) the
// overflowing pairs are also written to an exact spill list.
//
// Extra traffic against a direct probe: pairs written and read (16 B/key),
// all sequential.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "probe.cuh"

namespace dtlg {

constexpr uint32_t kPartTile = 4096;                    // keys per scatter tile
constexpr int kPartThreads = 512;                       // scatter CTA: 8 keys (2 key vectors) per thread
constexpr int kMaxRanges = 64;
constexpr uint32_t kPartChunk = 2048;                   // pairs per chunk of a segment
constexpr uint32_t kPartHeaderBytes = 512;              // fill counters + overflow counters

// Pairs the partition of n keys may need in all: the sum of the segment
// capacities (share + share/32 + one tile, rounded up to a chunk, per range).
__host__ __device__ constexpr uint64_t part_pair_capacity(uint64_t n) {
  return n + n / 32 + static_cast<uint64_t>(kMaxRanges) * (kPartTile + kPartChunk);
}

// Header of the partition's workspace (zeroed before the scatter).
struct PartHeader {
  unsigned int fill[kMaxRanges];     // pairs requested per range (may exceed the capacity)
  unsigned int overflow_tiles;       // tiles with at least one overflowing run
  unsigned int spill_cnt;            // pairs in the spill list
  unsigned int chunk_ctr;            // next chunk of the segments to hand out (pair kernels)
};
static_assert(sizeof(PartHeader) <= kPartHeaderBytes, "partition header");

struct PartArgs {
  const uint32_t* keys_al;  // 16-byte aligned key base (see ProbeArgs)
  uint64_t n_phys;
  uint32_t pre;
  Addr addr;
  uint32_t range_log2;      // a range is 2^range_log2 consecutive blocks
  uint32_t n_ranges;
  uint32_t n_tiles;
  uint32_t block_mul;       // the family constant of the block hash (C[0]; C[1]: blocked cuckoo)
  uint64_t seg_cap;         // capacity of every segment but the last (multiple of kPartChunk)
  uint64_t last_cap;        // capacity of the last segment (multiple of kPartChunk)
  uint2* pairs;             // (key, logical position); segment r starts at r * seg_cap
  PartHeader* hdr;
  unsigned long long* tile_overflow;  // [n_tiles]: bit r = the tile's run of range r overflowed
  uint2* spill;             // optional: every overflowing pair (capacity n_phys)
};

// Host-side sizing of the segments for n keys over `blocks` blocks in ranges
// of 2^range_log2 blocks.
inline void part_segments(uint64_t n, uint64_t blocks, uint32_t range_log2, uint32_t n_ranges, uint64_t* seg_cap,
                          uint64_t* last_cap) {
  auto cap = [&](uint64_t range_blocks) {
    const uint64_t share = (n * range_blocks + blocks - 1) / blocks;
    const uint64_t c = share + share / 32 + kPartTile;
    return (c + kPartChunk - 1) / kPartChunk * kPartChunk;
  };
  const uint64_t full = 1ull << range_log2;
  *seg_cap = cap(full < blocks ? full : blocks);
  *last_cap = cap(blocks - static_cast<uint64_t>(n_ranges - 1) * full);
}

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t key_range(uint32_t key, const PartArgs& a) {
  return block_index(key * a.block_mul, a.addr) >> a.range_log2;
}

// key_range with the addressing mode fixed at compile time (block_index
// branches on it at run time).
template <bool MAGIC>
__device__ __forceinline__ uint32_t key_range_of(uint32_t key, const PartArgs& a) {
  return block_index_of<MAGIC>(key * a.block_mul, a.addr) >> a.range_log2;
}

// Shared memory of one scatter CTA.
struct ScatterSmem {
  unsigned long long kv[kPartTile];    // the tile sorted by range: key | tile-local index << 32
  uint32_t cur[kMaxRanges];            // counts, then the placement cursor
  uint32_t lim[kMaxRanges];            // sorted slots below this go to the segment, the rest overflow
  unsigned long long dst[kMaxRanges];  // pair index of sorted slot 0 for the range's run
  uint32_t valid;
  unsigned long long over;
};

// One pass: per tile, count the keys of every range, reserve the tile's run of
// each range in its segment (one global atomic per tile and range), sort the
// tile by range in shared memory and write every run with consecutive
// addresses.  Shared memory holds the sorted keys with their 12-bit tile
// positions, one 64-bit word each (32 KiB).  The kernel is bound by instruction issue, so the
// addressing mode is a template parameter (POW2 or MAGIC, chosen by the
// launch), the tile's index arithmetic is 32-bit, a key's range is computed
// once for the count and the placement (kept as bytes), and each range's
// destination base and slot limit are computed once per tile.  512 threads of
// 8 keys each, four CTAs per SM (2^28 keys over 64 ranges of a 512 MiB POW2
// filter: 959 us with 256 threads of 16 keys and run-time addressing, 896 us
// so).
template <bool MAGIC, int THREADS>
__device__ __forceinline__ void scatter_tile(const PartArgs& a, uint32_t tile, ScatterSmem& S) {
  constexpr int kVecs = static_cast<int>(kPartTile) / THREADS / 4;  // key vectors per thread
  static_assert(kVecs * 4 * THREADS == static_cast<int>(kPartTile), "tile");
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t tile_pos = static_cast<uint64_t>(tile) * kPartTile;  // physical index of the tile's key 0
  // valid keys of this tile: tile-local indexes [lo, hi)
  const uint32_t lo = tile_pos < a.pre ? static_cast<uint32_t>(a.pre - tile_pos) : 0u;
  const uint32_t hi = a.n_phys - tile_pos < kPartTile ? static_cast<uint32_t>(a.n_phys - tile_pos) : kPartTile;
  const uint4* t4 = reinterpret_cast<const uint4*>(a.keys_al) + tile_pos / 4;
  // the keys are read twice: for the counts and, from L2, for the placement
  // (holding them across the scan would not fit 32 registers); their ranges
  // are kept, four bytes per register
  uint32_t rr[kVecs];
  {
    uint4 kv[kVecs];
#pragma unroll
    for (int i = 0; i < kVecs; i++) {
      const uint32_t li = (i * THREADS + threadIdx.x) * 4;
      kv[i] = li < hi ? __ldcg(t4 + li / 4) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int i = 0; i < kVecs; i++) {
      const uint32_t li = (i * THREADS + threadIdx.x) * 4;
      const uint32_t k[4] = {kv[i].x, kv[i].y, kv[i].z, kv[i].w};
      rr[i] = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint32_t r = key_range_of<MAGIC>(k[q], a);
        rr[i] |= r << (8 * q);
        if (li + q >= lo && li + q < hi) atomicAdd(&S.cur[r], 1u);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    // tile-local run starts (exclusive scan, two ranges per lane), the runs'
    // slots in their segments, and per range the destination of sorted slot
    // 0 and the first sorted slot that no longer fits the segment
    const uint32_t r0 = lane * 2, r1 = lane * 2 + 1;
    const uint32_t c0 = S.cur[r0], c1 = S.cur[r1];
    const uint32_t pair = c0 + c1;
    uint32_t incl = pair;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t x = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= static_cast<uint32_t>(d)) incl += x;
    }
    const uint32_t b0 = incl - pair;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uint32_t r = h ? r1 : r0, c = h ? c1 : c0, lb = h ? b0 + c0 : b0;
      const uint32_t g = c ? atomicAdd(&a.hdr->fill[r], c) : 0u;
      const uint64_t cap = r + 1 < a.n_ranges ? a.seg_cap : a.last_cap;
      const uint64_t room = g < cap ? cap - g : 0;
      S.cur[r] = lb;
      S.lim[r] = lb + static_cast<uint32_t>(room < c ? room : c);
      S.dst[r] = static_cast<uint64_t>(r) * a.seg_cap + g - lb;
    }
    if (lane == 31) S.valid = incl;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kVecs; i++) {
    const uint32_t li = (i * THREADS + threadIdx.x) * 4;
    const uint4 x = li < hi ? __ldcs(t4 + li / 4) : make_uint4(0, 0, 0, 0);
    const uint32_t k[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (li + q >= lo && li + q < hi) {
        const uint32_t slot = atomicAdd(&S.cur[(rr[i] >> (8 * q)) & 0xffu], 1u);
        S.kv[slot] = static_cast<unsigned long long>(li + q) << 32 | k[q];
      }
    }
  }
  __syncthreads();
  // the placement cursors are not read below: clear them for the next tile
  // (the barrier after the write-out orders this before its counts)
  if (threadIdx.x < kMaxRanges) S.cur[threadIdx.x] = 0;
  const uint32_t nv = S.valid;
  const uint32_t pos0 = static_cast<uint32_t>(tile_pos - a.pre);  // logical position of tile index 0 (mod 2^32)
  for (uint32_t sl = threadIdx.x; sl < nv; sl += THREADS) {
    const unsigned long long kv = S.kv[sl];
    const uint32_t key = static_cast<uint32_t>(kv);
    const uint32_t r = key_range_of<MAGIC>(key, a);
    const uint2 pr = make_uint2(key, pos0 + static_cast<uint32_t>(kv >> 32));
    if (sl < S.lim[r]) {
      __stcs(a.pairs + (S.dst[r] + sl), pr);
    } else {
      atomicOr(&S.over, 1ull << r);
      if (a.spill) a.spill[atomicAdd(&a.hdr->spill_cnt, 1u)] = pr;
    }
  }
  __syncthreads();
}

template <bool MAGIC, int THREADS = kPartThreads>
static __global__ void __launch_bounds__(THREADS, 2048 / THREADS) part_scatter_kernel(const __grid_constant__ PartArgs a) {
  __shared__ ScatterSmem S;
  // The counters start at zero; each tile clears them again for the next one
  // while it writes its runs out, so a tile needs no barrier of its own for it.
  if (threadIdx.x < kMaxRanges) S.cur[threadIdx.x] = 0;
  if (threadIdx.x == 0) S.over = 0;
  __syncthreads();
  for (uint32_t tile = blockIdx.x; tile < a.n_tiles; tile += gridDim.x) {
    scatter_tile<MAGIC, THREADS>(a, tile, S);
    if (threadIdx.x == 0) {
      // S.over is next written in the next tile's write-out, three barriers on
      a.tile_overflow[tile] = S.over;
      if (S.over) atomicAdd(&a.hdr->overflow_tiles, 1u);
      S.over = 0;
    }
  }
}

// The segments as a list of chunks of kPartChunk pairs, in range order.
struct SegChunks {
  const uint2* pairs;
  uint64_t seg_cap, last_cap;
  uint32_t n_ranges;
  uint32_t chunks_per_seg;  // seg_cap / kPartChunk (a segment holds < 2^32 pairs)
  uint32_t n_chunks;        // (n_ranges - 1) * chunks_per_seg + last_cap / kPartChunk
  const PartHeader* hdr;
};

__host__ __device__ inline SegChunks seg_chunks(const PartArgs& pa) {
  SegChunks s{};
  s.pairs = pa.pairs;
  s.seg_cap = pa.seg_cap;
  s.last_cap = pa.last_cap;
  s.n_ranges = pa.n_ranges;
  s.chunks_per_seg = static_cast<uint32_t>(pa.seg_cap / kPartChunk);
  s.n_chunks = (pa.n_ranges - 1) * s.chunks_per_seg + static_cast<uint32_t>(pa.last_cap / kPartChunk);
  s.hdr = pa.hdr;
  return s;
}

// Runs chunk(q, cnt) for every non-empty chunk of the segments (q: its pairs
// as 16-byte vectors of two, cnt: its pairs): CTAs take whole chunks from a
// queue (one atomic per chunk), in range order, so the chunks in flight are
// the ones next to each other and the filter range they read stays in L2 (a
// fixed grid-stride assignment lets slow and fast CTAs drift apart over two
// or more ranges, whose words then evict each other).  The ranges' fill
// counts are read into shared memory once per CTA.  The queue counter
// (PartHeader::chunk_ctr) must be zero.
template <class Chunk>
__device__ __forceinline__ void for_each_chunk(const SegChunks& s, Chunk chunk) {
  __shared__ uint32_t s_filled[kMaxRanges];  // pairs in each segment (fill, capped at the capacity)
  __shared__ uint32_t s_chunk;
  for (uint32_t r = threadIdx.x; r < s.n_ranges; r += blockDim.x) {
    const uint64_t cap = r + 1 < s.n_ranges ? s.seg_cap : s.last_cap;
    const uint32_t fill = s.hdr->fill[r];
    s_filled[r] = fill < cap ? fill : static_cast<uint32_t>(cap);
  }
  const uint4* p4 = reinterpret_cast<const uint4*>(s.pairs);
  const uint64_t half_seg = s.seg_cap >> 1;  // 16-byte vectors per segment
  unsigned int* ctr = const_cast<unsigned int*>(&s.hdr->chunk_ctr);
  for (;;) {
    if (threadIdx.x == 0) s_chunk = atomicAdd(ctr, 1u);
    __syncthreads();
    const uint32_t c = s_chunk;
    __syncthreads();  // s_chunk is rewritten for the next chunk
    if (c >= s.n_chunks) break;
    uint32_t r = c / s.chunks_per_seg;
    if (r >= s.n_ranges) r = s.n_ranges - 1;
    const uint32_t j0 = (c - r * s.chunks_per_seg) * kPartChunk;
    const uint32_t filled = s_filled[r];
    if (filled <= j0) continue;
    const uint32_t cnt = filled - j0 < kPartChunk ? filled - j0 : kPartChunk;
    chunk(p4 + static_cast<uint64_t>(r) * half_seg + (j0 >> 1), cnt);
  }
}

// fn(key, position) for every pair of the segments, two pairs per 16-byte load.
template <class Fn>
__device__ __forceinline__ void for_each_pair(const SegChunks& s, Fn fn) {
  for_each_chunk(s, [&](const uint4* q, uint32_t cnt) {
    for (uint32_t v = threadIdx.x; 2 * v < cnt; v += blockDim.x) {
      const uint4 x = __ldcs(q + v);
      fn(x.x, x.y);
      if (2 * v + 1 < cnt) fn(x.z, x.w);
    }
  });
}

// for_each_pair for warp-cooperative callbacks: every lane of the CTA calls
// fn(key, valid) the same number of times (valid = false past the chunk's end).
template <class Fn>
__device__ __forceinline__ void for_each_pair_warp(const SegChunks& s, Fn fn) {
  for_each_chunk(s, [&](const uint4* q, uint32_t cnt) {
    for (uint32_t vb = 0; 2 * vb < cnt; vb += blockDim.x) {
      const uint32_t v = vb + threadIdx.x;
      const uint4 x = 2 * v < cnt ? __ldcs(q + v) : make_uint4(0, 0, 0, 0);
      fn(x.x, 2 * v < cnt);
      fn(x.z, 2 * v + 1 < cnt);
    }
  });
}

// Runs fn(key, logical position) over the keys of every tile whose run of the
// key's range overflowed its segment (all keys of that range in that tile,
// the ones that did fit included); nothing when no tile overflowed.
template <class Fn>
__device__ __forceinline__ void for_each_overflow_key(const PartArgs& pa, Fn fn) {
  if (pa.hdr->overflow_tiles == 0) return;
  const uint4* keys4 = reinterpret_cast<const uint4*>(pa.keys_al);
  for (uint32_t tile = blockIdx.x; tile < pa.n_tiles; tile += gridDim.x) {
    const unsigned long long mask = pa.tile_overflow[tile];
    if (mask == 0) continue;
    const uint64_t v0 = static_cast<uint64_t>(tile) * (kPartTile / 4);
    for (uint32_t i = threadIdx.x; i < kPartTile / 4; i += blockDim.x) {
      const uint64_t v = v0 + i;
      if (v * 4 >= pa.n_phys) break;
      const uint4 kv = keys4[v];
      const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint64_t p = v * 4 + q;
        if (p >= pa.pre && p < pa.n_phys && ((mask >> key_range(k[q], pa)) & 1ull))
          fn(k[q], static_cast<uint32_t>(p - pa.pre));
      }
    }
  }
}

struct PairsArgs {
  ProbeArgs probe;          // filter + addressing (keys fields unused)
  PartArgs part;            // the partition the pairs came from
  uint32_t* bits;           // key-ordered match mask (bit = physical key index), zeroed
  uint32_t pre;             // physical index of the first key
};

template <class Ops>
__device__ __forceinline__ void probe_pair(const PairsArgs& a, uint32_t key, uint32_t pos) {
  if (Ops::contains(a.probe, key)) {
    const uint64_t b = static_cast<uint64_t>(pos) + a.pre;
    atomicOr(a.bits + (b >> 5), 1u << (b & 31u));
  }
}

// Probes the pairs in range order; each match sets one bit of the mask.
template <class Ops, int MINB>
__global__ void __launch_bounds__(256, MINB) probe_pairs_kernel(const __grid_constant__ PairsArgs a) {
  for_each_pair(seg_chunks(a.part), [&](uint32_t key, uint32_t pos) { probe_pair<Ops>(a, key, pos); });
}

// The keys of overflowing runs, after probe_pairs_kernel: a kernel of its
// own, so that the pair kernel's register budget holds only its loop.  When
// no segment filled up (the rule for hashed keys) every CTA returns at once.
template <class Ops>
__global__ void __launch_bounds__(256) probe_overflow_kernel(const __grid_constant__ PairsArgs a) {
  for_each_overflow_key(a.part, [&](uint32_t key, uint32_t pos) { probe_pair<Ops>(a, key, pos); });
}

#endif  // __CUDACC__

}  // namespace dtlg
