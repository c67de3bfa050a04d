// bcf.cuh -- blocked cuckoo filter probe and build (dtl::bcf).
//
// Reference: bcf.hpp:11-63 / bcf.cpp over blocked_cuckoofilter/*.hpp.  The
// filter is an array of blocks of 8..512 bytes; every block is a small
// partial-key cuckoo table of one-word buckets (all configs the dispatcher
// offers, blocked_cuckoofilter.hpp:254-297, hold exactly one bucket per word:
// u64 words for t*a > 32 bits, u32 words otherwise).  A key touches one block:
//
//   h   = key * C[1]                         block = addr(h)   (logic.hpp:73-76)
//   hv  = h << log2(B)   (POW2, when log2(B) + t + log2(buckets) <= 32)
//       = key * C[0]     (otherwise: MAGIC, or too few bits left; :77-82)
//   i1  = hv >> (32 - bb)                    (block_logic.hpp:45-49; bb = log2(buckets))
//   tag = (hv >> (32 - bb - t)) & mask, 0 -> 1                              (:128-133)
//   i2  = i1 ^ ((tag * 0x5bd1e995) >> (32 - bb))                            (:69-72)
//
// contains = either bucket overflowed (all tag bits set) or holds the tag,
// tested with the reference's SWAR field test (blocked_cuckoofilter_util.hpp:
// 14-88, multiword_table.hpp:51-67).  That is the reference's scalar path;
// its AVX2 batch path of <16,4> and <8,4> also reports keys whose bucket holds
// any all-ones tag field, a superset not reproduced here.
//
// Build: the reference inserts key after key; a full bucket swaps the tag
// with a random slot (thread-local mt19937) and after 10 relocations marks
// the last bucket as overflowed (block_logic.hpp:96-118), so no two of its
// builds agree.  Here every key is inserted by its own thread; each step of
// the algorithm reads one bucket word and replaces it with a compare-and-swap,
// retried on a lost race.  A thread that holds a displaced tag carries it on,
// as the sequential code does, so every key ends in one of its two buckets or
// behind an overflowed bucket: no false negatives.
#pragma once

#include <cstdint>
#include <type_traits>

#include "bloom.cuh"
#include "common.cuh"
#include "probe.cuh"

namespace dtlg {

template <int T, int A>
struct BcfCfg {
  static constexpr int kT = T, kA = A;
  static constexpr int kBucketBits = T * A;
  static constexpr bool kWide = kBucketBits > 32;  // u64 words
  using word_t = typename std::conditional<kWide, unsigned long long, unsigned int>::type;
  static constexpr int kWordBits = kWide ? 64 : 32;
  static constexpr uint32_t kTagMask = (1u << T) - 1u;
  // multiword_table.hpp:100,111: a bucket whose tag bits are all set
  static constexpr unsigned long long kOverflow =
      kBucketBits == 64 ? ~0ull : ((1ull << kBucketBits) - 1ull);
  // SWAR field sets of packed_value<word, T> (blocked_cuckoofilter_util.hpp):
  // fields of T bits at 0, T, 2T, ...; with 16-bit tags in 32-bit words the
  // reference's constants are 64-bit, so that test runs on 64 bits.
  static constexpr int kFields = T == 8 ? kWordBits / 8 : (T == 10 ? 6 : (T == 12 ? 5 : 4));
  static constexpr bool kSwar32 = (T == 8 && !kWide);
  static constexpr unsigned long long swar_low() {
    unsigned long long l = 0;
    for (int i = 0; i < kFields; i++) l |= 1ull << (T * i);
    return l;
  }
  static constexpr unsigned long long kLow = swar_low();
  static constexpr unsigned long long kHigh = kLow << (T - 1);
};

struct BcfBuildArgs {
  void* filter;
  const uint32_t* keys_al;
  uint64_t n_phys;
  uint32_t pre;
  Addr addr;
  uint32_t bucket_bits;   // log2(buckets per block)
  uint32_t hash_shift;    // < 32: bucket hash = block hash << hash_shift; 32: key * C[0]
  uint64_t seed;
};

constexpr uint32_t kBcfAltMul = 0x5bd1e995u;  // block_logic.hpp:71
constexpr uint32_t kBcfRelocations = 10;     // block_logic.hpp:108
constexpr uint32_t kBcfCasLimit = 1u << 16;  // lost races tolerated per step

#ifdef __CUDACC__

template <class Cfg>
struct BcfOps {
  using Word = typename Cfg::word_t;

  // packed_value<word, T>::contains: does any field equal n (n != 0)?
  __device__ __forceinline__ static bool has(Word x, uint32_t n) {
    if constexpr (Cfg::kSwar32) {
      const uint32_t L = static_cast<uint32_t>(Cfg::kLow), H = static_cast<uint32_t>(Cfg::kHigh);
      const uint32_t y = static_cast<uint32_t>(x) ^ (n * L);
      return ((y - L) & ~y & H) != 0u;
    } else {
      const unsigned long long y = static_cast<unsigned long long>(x) ^ (static_cast<unsigned long long>(n) * Cfg::kLow);
      return ((y - Cfg::kLow) & ~y & Cfg::kHigh) != 0ull;
    }
  }

  // Block, bucket hash (logic.hpp:73-82).
  __device__ __forceinline__ static uint32_t block_hash(uint32_t key, const Addr& a, uint32_t hash_shift,
                                                        uint32_t& hv) {
    const uint32_t h = key * mul_const(1);
    hv = hash_shift < 32u ? (h << hash_shift) : key * mul_const(0);
    return block_index(h, a);
  }

  // Bucket pair and tag inside the block (block_logic.hpp:45-72,128-133);
  // 64-bit shifts make a block of one bucket (bb = 0) give index 0.
  __device__ __forceinline__ static void bucket_tag(uint32_t hv, uint32_t bb, uint32_t& i1, uint32_t& i2,
                                                    uint32_t& tag) {
    i1 = static_cast<uint32_t>(static_cast<unsigned long long>(hv) >> (32u - bb));
    tag = (hv >> (32u - bb - Cfg::kT)) & Cfg::kTagMask;
    tag += (tag == 0u);
    i2 = i1 ^ static_cast<uint32_t>(static_cast<unsigned long long>(tag * kBcfAltMul) >> (32u - bb));
  }

  __device__ __forceinline__ static uint32_t alt(uint32_t i, uint32_t tag, uint32_t bb) {
    return i ^ static_cast<uint32_t>(static_cast<unsigned long long>(tag * kBcfAltMul) >> (32u - bb));
  }

  // Word j (< words per 32-byte sector) of a sector held as four u64.
  __device__ __forceinline__ static Word pick(const unsigned long long (&v)[4], uint32_t j) {
    if constexpr (Cfg::kWide) {
      return j == 0 ? v[0] : (j == 1 ? v[1] : (j == 2 ? v[2] : v[3]));
    } else {
      const unsigned long long x = (j >> 1) == 0 ? v[0] : ((j >> 1) == 1 ? v[1] : ((j >> 1) == 2 ? v[2] : v[3]));
      return static_cast<Word>(x >> (32u * (j & 1u)));
    }
  }

  // The two bucket words of a block.  Every load of a random address costs an
  // L1 lookup of its own, so blocks of >= 32 bytes on a 32-byte aligned filter
  // read the 32-byte sector of the first bucket with one 256-bit load and
  // fetch the second word separately only when it lies in another sector
  // (half the keys in a 64-byte block); a one-word block is read once.
  __device__ __forceinline__ static void load_pair(const Word* p, uint32_t i1, uint32_t i2, uint32_t bb,
                                                   bool vec32, Word& w1, Word& w2) {
    constexpr uint32_t kWps = 32u / sizeof(Word);  // words per 32-byte sector
    constexpr uint32_t kLwps = sizeof(Word) == 8 ? 2u : 3u;
    if (vec32 && bb >= kLwps) {
      const uint32_t s1 = i1 >> kLwps;
      unsigned long long v[4];
      ld_nc_256(p + (s1 << kLwps), v[0], v[1], v[2], v[3]);
      w1 = pick(v, i1 & (kWps - 1u));
      w2 = (i2 >> kLwps) == s1 ? pick(v, i2 & (kWps - 1u)) : __ldg(p + i2);
    } else if (bb == 0) {
      w1 = w2 = __ldg(p);
    } else {
      w1 = __ldg(p + i1);
      w2 = __ldg(p + i2);
    }
  }

  __device__ __forceinline__ static bool contains(const ProbeArgs& a, uint32_t key) {
    uint32_t hv;
    const uint32_t blk = block_hash(key, a.addr, a.bcf_hash_shift, hv);
    if (a.range_on && (blk < a.blk_lo || blk >= a.blk_hi)) return false;  // another pass's block
    uint32_t i1, i2, tag;
    bucket_tag(hv, a.bcf_bucket_bits, i1, i2, tag);
    const Word* p = static_cast<const Word*>(a.filter) + (static_cast<uint64_t>(blk) << a.bcf_bucket_bits);
    Word w1, w2;
    load_pair(p, i1, i2, a.bcf_bucket_bits, a.vec32 != 0u, w1, w2);
    return (w1 == static_cast<Word>(Cfg::kOverflow)) | (w2 == static_cast<Word>(Cfg::kOverflow)) | has(w1, tag) |
           has(w2, tag);
  }
};

__device__ __forceinline__ uint32_t bcf_rand(uint64_t& s) {  // xorshift64* (Vigna 2014)
  s ^= s >> 12;
  s ^= s << 25;
  s ^= s >> 27;
  return static_cast<uint32_t>((s * 2685821657736338717ull) >> 32);
}

__device__ __forceinline__ unsigned int bcf_cas(unsigned int* p, unsigned int c, unsigned int v) {
  return atomicCAS(p, c, v);
}
__device__ __forceinline__ unsigned long long bcf_cas(unsigned long long* p, unsigned long long c,
                                                      unsigned long long v) {
  return atomicCAS(p, c, v);
}
__device__ __forceinline__ unsigned int bcf_load(const unsigned int* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned long long bcf_load(const unsigned long long* p) { return __ldcg(p); }

constexpr uint32_t kBcfPlaced = 0u;             // stored, or already present
constexpr uint32_t kBcfOverflowed = 0xFFFFFFFFu;  // the bucket is overflowed

// insert_tag / insert_tag_relocate (multiword_table.hpp:176-224) as one
// compare-and-swap step on the bucket word: the first slot holding the tag or
// empty takes it; a full bucket returns `tag` (no relocation) or swaps it
// into a random slot and returns the tag it displaced.  A step that keeps
// losing races marks the bucket overflowed, which answers every key of it.
template <class Cfg>
__device__ __forceinline__ uint32_t bcf_insert_tag(typename Cfg::word_t* w, uint32_t tag, bool relocate,
                                                   uint64_t& rng) {
  using Word = typename Cfg::word_t;
  constexpr Word kOvf = static_cast<Word>(Cfg::kOverflow);
  Word cur = bcf_load(w);
  for (uint32_t tries = 0; tries < kBcfCasLimit; tries++) {
    if (cur == kOvf) return kBcfOverflowed;
    Word next = cur;
    uint32_t out = kBcfPlaced;
    bool write = false, done = false;
#pragma unroll
    for (int j = 0; j < Cfg::kA; j++) {
      if (done) continue;
      const uint32_t x = static_cast<uint32_t>(cur >> (Cfg::kT * j)) & Cfg::kTagMask;
      if (x == tag) {
        done = true;
      } else if (x == 0u) {
        next = cur | (static_cast<Word>(tag) << (Cfg::kT * j));
        write = done = true;
      }
    }
    if (!done) {
      if (!relocate) return tag;
      const uint32_t r = bcf_rand(rng) % Cfg::kA;
      out = static_cast<uint32_t>(cur >> (Cfg::kT * r)) & Cfg::kTagMask;
      next = cur ^ (static_cast<Word>(out ^ tag) << (Cfg::kT * r));
      write = true;
    }
    if (!write) return kBcfPlaced;
    const Word seen = bcf_cas(w, cur, next);
    if (seen == cur) return out;
    cur = seen;
  }
  atomicExch(w, kOvf);
  return kBcfOverflowed;
}

// blocked_cuckoofilter_logic.hpp:73-95 with block_logic.hpp:96-118 for one
// key; idx seeds the key's kick-slot generator.
template <class Cfg>
__device__ __forceinline__ void bcf_insert_key(const BcfBuildArgs& a, uint32_t key, uint64_t idx) {
  using Word = typename Cfg::word_t;
  using Ops = BcfOps<Cfg>;
  const uint32_t bb = a.bucket_bits;
  uint32_t hv, i1, i2, tag;
  const uint32_t blk = Ops::block_hash(key, a.addr, a.hash_shift, hv);
  Ops::bucket_tag(hv, bb, i1, i2, tag);
  Word* block = static_cast<Word*>(a.filter) + (static_cast<uint64_t>(blk) << bb);
  uint64_t rng = a.seed ^ (0x9E3779B97F4A7C15ull * (idx + 1));
  uint32_t old = bcf_insert_tag<Cfg>(block + i1, tag, false, rng);
  if (old == kBcfPlaced || old == kBcfOverflowed) return;
  uint32_t cur = i2, cur_tag = tag;
  for (uint32_t c = 0; c < kBcfRelocations; c++) {
    old = bcf_insert_tag<Cfg>(block + cur, cur_tag, true, rng);
    if (old == kBcfPlaced || old == kBcfOverflowed) return;
    cur_tag = old;
    cur = Ops::alt(cur, cur_tag, bb);
  }
  atomicExch(block + cur, static_cast<Word>(Cfg::kOverflow));  // mark_overflow
}

// One key per thread.
template <class Cfg>
__global__ void __launch_bounds__(256) bcf_insert_kernel(const __grid_constant__ BcfBuildArgs a) {
  for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < a.n_phys;
       p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    if (p < a.pre) continue;
    bcf_insert_key<Cfg>(a, __ldg(a.keys_al + p), p);
  }
}

// The same over range-grouped (key, position) pairs (probe3.cuh's
// partition): consecutive keys hit the same L2-sized block range, so the
// compare-and-swap steps of a filter far larger than L2 work on lines in L2.
// A second insert of a key would take a second slot, so the keys whose run
// overflowed its segment come from the partition's exact spill list.
template <class Cfg>
__global__ void __launch_bounds__(256) bcf_insert_pairs_kernel(const __grid_constant__ BcfBuildArgs a,
                                                               const __grid_constant__ PartArgs pa) {
  for_each_pair(seg_chunks(pa), [&](uint32_t key, uint32_t pos) { bcf_insert_key<Cfg>(a, key, pos); });
  const uint32_t n_spill = pa.hdr->spill_cnt;
  for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < n_spill;
       p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint2 x = pa.spill[p];
    bcf_insert_key<Cfg>(a, x.x, x.y);
  }
}

#endif  // __CUDACC__

}  // namespace dtlg
