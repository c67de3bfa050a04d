// probe2.cuh -- batch_contains as two streaming kernels, for large batches.
//
// 1. probe_bits_kernel: every warp takes chunks of 128 keys (one 16-byte key
//    vector per lane), tests them, and writes the 128 match flags as four
//    32-bit words of a key-ordered bitmask.  No barrier, no look-back: the only
//    thing a warp ever waits for is its own filter loads.  probe_smem_kernel
//    does the same against a copy of a small filter in shared memory.
// 2. compact_kernel: turns the bitmask into the ascending position list.  A
//    tile is 65536 keys (2048 mask words); the tile offset comes from a
//    decoupled look-back (bounded waits, as in probe.cuh) over a few thousand
//    status words.  It moves 1/8 byte per key in and 4 bytes per match out,
//    staged per warp in shared memory so the stores are coalesced.
// The extra traffic against the fused kernel is the bitmask, 2/8 byte per key.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "probe.cuh"

namespace dtlg {

constexpr int kCompactThreads = 256;
constexpr int kCompactWordsPerThread = 8;
constexpr uint32_t kCompactTileWords = kCompactThreads * kCompactWordsPerThread;
constexpr uint32_t kMaxGatherCols = 4;

struct CompactArgs {
  const uint32_t* bits;        // key-ordered match bitmask (bit i = physical key i)
  uint64_t n_words;            // ceil(n_phys / 32)
  uint32_t pre;                // physical index of the first key
  uint32_t match_offset;
  uint32_t* out;
  unsigned long long* count_out;
  unsigned long long* status;  // per-tile look-back words (zeroed)
  unsigned int* tile_ctr;      // zeroed
  unsigned int* err;           // zeroed
  uint32_t n_tiles;
  // probe -> gather: with every match i (logical index) written to slot j of
  // the list, row i of each payload column goes to row j of its output column
  uint32_t n_cols;             // 0 .. kMaxGatherCols
  uint32_t col_bytes[kMaxGatherCols];  // 4 or 8
  const void* cols[kMaxGatherCols];
  void* out_cols[kMaxGatherCols];
};

#ifdef __CUDACC__

// The bitmask loop: every warp takes chunks of 128 keys (one 16-byte key
// vector per lane), tests them with test(key) and writes the 128 flags as four
// 32-bit words of the key-ordered mask.  or_into: a later block-range pass ORs
// its flags into the words of the earlier passes (every word is written by
// exactly one warp per pass, and the passes are ordered on one stream).
template <class Test>
__device__ __forceinline__ void bits_loop(const ProbeArgs& a, uint32_t* __restrict__ bits, int or_into,
                                          Test test) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint4* keys4 = reinterpret_cast<const uint4*>(a.keys_al);
  const uint64_t n_vec = (a.n_phys + 3) >> 2;
  const uint64_t n_words = (a.n_phys + 31) >> 5;
  const uint64_t n_chunks = (n_vec + 31) >> 5;  // 32 key vectors = 128 keys
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t c = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); c < n_chunks;
       c += warps) {
    const uint64_t v = c * 32 + lane;
    uint32_t f = 0;
    if (v < n_vec) {
      const uint4 kv = __ldcs(keys4 + v);
      const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
      for (int q = 0; q < 4; q++) f |= (test(k[q]) ? 1u : 0u) << q;
      const uint64_t p0 = v * 4;
      if (p0 < a.pre || p0 + 4 > a.n_phys) {
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (p0 + q < a.pre || p0 + q >= a.n_phys) f &= ~(1u << q);
      }
    }
    // lanes 8j .. 8j+7 hold keys 32j .. 32j+31 of the chunk: word j
    uint32_t x = f << (4u * (lane & 7u));
    x |= __shfl_xor_sync(0xffffffffu, x, 1);
    x |= __shfl_xor_sync(0xffffffffu, x, 2);
    x |= __shfl_xor_sync(0xffffffffu, x, 4);
    if ((lane & 7u) == 0) {
      const uint64_t w = c * 4 + (lane >> 3);
      if (w < n_words) {
        if (or_into) x |= __ldcg(bits + w);
        __stcg(bits + w, x);
      }
    }
  }
}

template <class Ops, int MINB>
__global__ void __launch_bounds__(256, MINB)
probe_bits_kernel(const __grid_constant__ ProbeArgs a, uint32_t* __restrict__ bits, int or_into) {
  bits_loop(a, bits, or_into, [&](uint32_t key) { return Ops::contains(a, key); });
}

// Plan 4, filters that fit in shared memory: every CTA first copies the whole
// filter (filter_words32 32-bit words) into shared memory with coalesced
// loads, then runs the bitmask loop against that copy.  Random block reads
// then cost shared-memory bank cycles instead of L1TEX tag lookups.
constexpr int kSmemThreads = 512;

template <class Ops>
__global__ void __launch_bounds__(kSmemThreads)
probe_smem_kernel(const __grid_constant__ ProbeArgs a, uint32_t* __restrict__ bits, uint32_t filter_words32) {
  extern __shared__ uint4 s_filter[];
  const uint32_t n_vec = filter_words32 >> 2;
  const uint4* g4 = static_cast<const uint4*>(a.filter);
  for (uint32_t i = threadIdx.x; i < n_vec; i += blockDim.x) s_filter[i] = __ldg(g4 + i);
  uint32_t* s32 = reinterpret_cast<uint32_t*>(s_filter);
  const uint32_t* g32 = static_cast<const uint32_t*>(a.filter);
  for (uint32_t i = n_vec * 4 + threadIdx.x; i < filter_words32; i += blockDim.x) s32[i] = __ldg(g32 + i);
  __syncthreads();
  bits_loop(a, bits, 0, [&](uint32_t key) { return Ops::contains_shared(s_filter, a, key); });
}

// Ordered compaction.  A tile is kCompactTileWords mask words; warp w of the
// CTA owns the 256 words w*256 .. w*256+255 of the tile as 8 rows of 32 words
// (lane l holds word i*32 + l of row i, so every row is one coalesced 128-byte
// load).  The tile's offset comes from the look-back; the warp's from a CTA
// scan; each row's from a warp scan.  A row's matches (at most 1024) are
// first written to a per-warp staging area in shared memory in key order and
// then stored by the whole warp to consecutive output slots, so the output
// (and the payload gathers) are coalesced however dense the matches are.
static __global__ void __launch_bounds__(kCompactThreads) compact_kernel(const __grid_constant__ CompactArgs a) {
  constexpr int kWarps = kCompactThreads / 32;
  constexpr int kRows = kCompactWordsPerThread;  // rows of 32 words per warp
  static_assert(kCompactTileWords == kWarps * kRows * 32, "tile = warps x rows x 32 words");
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kWarps];
  __shared__ uint32_t s_excl;
  __shared__ uint32_t s_stage[kWarps][1024];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = threadIdx.x >> 5;
  // the look-back helper of probe.cuh reads status / err from a ProbeArgs
  ProbeArgs lb{};
  lb.status = a.status;
  lb.err = a.err;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= a.n_tiles) break;
    const uint64_t wbase = static_cast<uint64_t>(tile) * kCompactTileWords + static_cast<uint64_t>(warp) * (kRows * 32);
    uint32_t wv[kRows];
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < kRows; i++) {
      const uint64_t idx = wbase + static_cast<uint64_t>(i) * 32 + lane;
      wv[i] = idx < a.n_words ? __ldcs(a.bits + idx) : 0u;
      c += __popc(wv[i]);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(0xffffffffu, c, d);
    if (lane == 0) s_warp[warp] = c;  // the warp's match count
    __syncthreads();
    if (warp == 0) {
      const uint32_t v = lane < kWarps ? s_warp[lane] : 0u;
      uint32_t wi = v;
#pragma unroll
      for (int d = 1; d < kWarps; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, wi, d);
        if (lane >= static_cast<uint32_t>(d)) wi += t;
      }
      const uint32_t agg = __shfl_sync(0xffffffffu, wi, kWarps - 1);
      if (lane < kWarps) s_warp[lane] = wi - v;
      uint32_t excl = 0;
      if (tile == 0) {
        if (lane == 0) st_volatile(a.status, kFlagPrefix | agg);
      } else {
        if (lane == 0) st_volatile(a.status + tile, kFlagAgg | agg);
        excl = look_back(lb, tile, lane);
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
    uint32_t pos = s_excl + s_warp[warp];
    uint32_t* stage = s_stage[warp];
#pragma unroll
    for (int i = 0; i < kRows; i++) {
      // the row's matches in key order: lanes in order, bits in order
      const uint32_t ci = __popc(wv[i]);
      uint32_t incl = ci;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= static_cast<uint32_t>(d)) incl += t;
      }
      const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
      if (tot == 0) continue;
      // logical index of bit 0 of this lane's word
      const uint32_t first = static_cast<uint32_t>((wbase + static_cast<uint64_t>(i) * 32 + lane) * 32 - a.pre);
      uint32_t m = wv[i];
      uint32_t o = incl - ci;
      while (m) {
        const uint32_t b = __ffs(m) - 1;
        m &= m - 1;
        stage[o++] = first + b;
      }
      __syncwarp();
      for (uint32_t j = lane; j < tot; j += 32) {
        const uint32_t li = stage[j];
        if (a.out) __stcs(a.out + pos + j, li + a.match_offset);
        for (uint32_t col = 0; col < a.n_cols; col++) {
          if (a.col_bytes[col] == 8) {
            __stcs(static_cast<unsigned long long*>(a.out_cols[col]) + pos + j,
                   __ldcs(static_cast<const unsigned long long*>(a.cols[col]) + li));
          } else {
            __stcs(static_cast<uint32_t*>(a.out_cols[col]) + pos + j,
                   __ldcs(static_cast<const uint32_t*>(a.cols[col]) + li));
          }
        }
      }
      __syncwarp();
      pos += tot;
    }
    __syncthreads();
  }
}

#endif  // __CUDACC__

}  // namespace dtlg
