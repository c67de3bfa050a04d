// cuckoo.cuh -- partial-key cuckoo filter probe and build.
//
// Reference: cuckoofilter_logic.hpp:119-521 and cuckoofilter_table.hpp:67-277.
// Table layout (identical bytes): buckets of ceil(T*B/8) bytes, tag j of a
// bucket at bit T*j (little endian), tag 0 = empty; the victim record
// {u32 index, u32 tag, bool used} follows the table at 32-bit word
// ceil(bytes/4) (cuckoofilter_logic.hpp:131-157).
//
// Probe: bit-exact with the reference (the reference's SWAR bucket tests,
// cuckoofilter_table_scalar.hpp:48-83, are exact existence tests).
//
// Build: the reference inserts one key at a time and picks kick slots with a
// thread-local mt19937 seeded from std::random_device (cuckoofilter_table.hpp:
// 197, thread.hpp:72-78), so no two of its builds agree.  The GPU build runs
// the same bounded-kick partial-key algorithm for all keys at once on an
// unpacked copy of the table (one 32-bit slot per tag, atomicCAS to claim an
// empty slot, atomicExch to kick), then packs it back into the reference
// layout.  Checked by invariants (no false negatives, occupancy) and FPR.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "probe.cuh"

namespace dtlg {

constexpr uint32_t kAltMul = 0x5bd1e995u;  // cuckoofilter_logic.hpp:222,246
constexpr uint32_t kMaxKicks = 500;        // cuckoofilter_logic.hpp:122

template <int T, int B>
struct CuckooCfg {
  static constexpr int kT = T, kB = B;
  static constexpr int kBytesPerBucket = (T * B + 7) / 8;
  static constexpr uint32_t kTagMask = T == 32 ? 0xffffffffu : ((1u << T) - 1u);
};

struct CuckooBuildArgs {
  uint32_t* table;          // packed table (32-bit words) + victim record
  uint32_t* slots;          // unpacked: (bucket_cnt + 1) * B slots
  const uint32_t* keys_al;
  uint64_t n_phys;
  uint32_t pre;
  uint64_t table_words;     // 32-bit words of the packed table
  uint64_t victim_word;
  Addr addr;
  unsigned long long* failed;  // keys whose tag could not be placed
  uint64_t seed;
};

#ifdef __CUDACC__

// Alternate bucket (cuckoofilter_logic.hpp:214-252).  The MAGIC form yields
// bucket_cnt (one past the end) for i == 0 and tag*M mod c == 0; the reference
// then reads the bytes after the table, and so does the probe here.
__device__ __forceinline__ uint32_t cuckoo_alt(uint32_t i, uint32_t tag, const Addr& a) {
  if (!a.magic_mode) return (i ^ (tag * kAltMul)) & a.block_cnt_mask;
  const uint32_t c = a.divisor;
  const uint32_t s = block_index(tag * kAltMul, a);
  const uint32_t x = c - s;
  return (x < i ? c : 0u) + (x - i);
}

template <class Cfg>
struct CuckooOps {
  static constexpr int kT = Cfg::kT, kB = Cfg::kB, kBPB = Cfg::kBytesPerBucket;

  __device__ __forceinline__ static void index_tag(uint32_t key, const Addr& a, uint32_t& i1,
                                                   uint32_t& tag) {
    i1 = block_index(key * mul_const(0), a);         // cuckoofilter_logic.hpp:205
    tag = (key * mul_const(1)) & Cfg::kTagMask;       // :183, :206
    tag += (tag == 0u);                          // :184
  }

  // Does bucket i hold `tag`?  Reads the bucket's bytes with aligned loads.
  __device__ __forceinline__ static bool bucket_has(const void* table, uint32_t i, uint32_t tag) {
    const uint64_t o = static_cast<uint64_t>(i) * kBPB;
    const unsigned char* t8 = static_cast<const unsigned char*>(table);
    bool hit = false;
    if constexpr (kBPB == 16) {
      const uint4 x = __ldg(reinterpret_cast<const uint4*>(t8 + o));
      hit = (x.x == tag) | (x.y == tag) | (x.z == tag) | (x.w == tag);
    } else if constexpr (kBPB == 8) {
      const unsigned long long x = __ldg(reinterpret_cast<const unsigned long long*>(t8 + o));
#pragma unroll
      for (int j = 0; j < kB; j++) hit |= ((x >> (kT * j)) & Cfg::kTagMask) == tag;
    } else if constexpr (kBPB == 4) {
      const uint32_t x = __ldg(reinterpret_cast<const unsigned int*>(t8 + o));
#pragma unroll
      for (int j = 0; j < kB; j++) hit |= ((x >> (kT * j)) & Cfg::kTagMask) == tag;
    } else {
      // 1, 2, 3 or 6 bytes: at most two aligned 32-bit words hold the bucket
      const uint64_t a4 = o & ~3ull;
      const uint32_t sh = static_cast<uint32_t>(o & 3u) * 8u;
      const unsigned int* w = reinterpret_cast<const unsigned int*>(t8 + a4);
      unsigned long long x = __ldg(w);
      if constexpr (kBPB > 2) x |= static_cast<unsigned long long>(__ldg(w + 1)) << 32;
#pragma unroll
      for (int j = 0; j < kB; j++) hit |= ((x >> (sh + kT * j)) & Cfg::kTagMask) == tag;
    }
    return hit;
  }

  // cuckoofilter_logic.hpp:346-362
  __device__ __forceinline__ static bool contains(const ProbeArgs& a, uint32_t key) {
    uint32_t i1, tag;
    index_tag(key, a.addr, i1, tag);
    const uint32_t i2 = cuckoo_alt(i1, tag, a.addr);
    const unsigned int* v = static_cast<const unsigned int*>(a.filter) + a.victim_word;
    const uint32_t vi = __ldg(v), vt = __ldg(v + 1), vu = __ldg(v + 2) & 0xffu;
    const bool in_victim = vu && tag == vt && (i1 == vi || i2 == vi);
    if (a.range_on) {
      // block-range pass: only the buckets this pass owns (the result is the OR
      // over all passes)
      const bool r1 = i1 >= a.blk_lo && i1 < a.blk_hi;
      const bool r2 = i2 >= a.blk_lo && i2 < a.blk_hi;
      return in_victim | (r1 && bucket_has(a.filter, i1, tag)) | (r2 && bucket_has(a.filter, i2, tag));
    }
    return in_victim | bucket_has(a.filter, i1, tag) | bucket_has(a.filter, i2, tag);
  }

  // cuckoofilter_table.hpp:111-136: tag j of bucket i from the packed table.
  __device__ __forceinline__ static uint32_t read_tag(const uint32_t* table, uint64_t i, int j) {
    const uint64_t bit = i * (kBPB * 8ull) + static_cast<uint64_t>(kT) * j;
    const uint64_t w = bit >> 5;
    const uint32_t sh = static_cast<uint32_t>(bit & 31u);
    unsigned long long x = table[w];
    if (sh + kT > 32) x |= static_cast<unsigned long long>(table[w + 1]) << 32;
    return static_cast<uint32_t>(x >> sh) & Cfg::kTagMask;
  }
};

template <class Cfg>
__global__ void cuckoo_unpack_kernel(const uint32_t* table, uint32_t* slots, uint32_t bucket_cnt) {
  const uint64_t n = static_cast<uint64_t>(bucket_cnt) * Cfg::kB;
  for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < n;
       s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    slots[s] = CuckooOps<Cfg>::read_tag(table, s / Cfg::kB, static_cast<int>(s % Cfg::kB));
  }
}

__device__ __forceinline__ uint32_t kick_rand(uint64_t& s) {  // xorshift64* (Vigna 2014)
  s ^= s >> 12;
  s ^= s << 25;
  s ^= s >> 27;
  return static_cast<uint32_t>((s * 2685821657736338717ull) >> 32);
}

// cuckoofilter_logic.hpp:292-322, all keys in parallel on the slot array.
template <class Cfg>
__global__ void __launch_bounds__(256) cuckoo_insert_kernel(const __grid_constant__ CuckooBuildArgs a) {
  constexpr int kB = Cfg::kB;
  const uint32_t c = a.addr.block_cnt;
  for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < a.n_phys;
       p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    if (p < a.pre) continue;
    const uint32_t key = __ldg(a.keys_al + p);
    uint32_t cur, tag;
    CuckooOps<Cfg>::index_tag(key, a.addr, cur, tag);
    uint64_t rng = a.seed ^ (0x9E3779B97F4A7C15ull * (p + 1));
    bool done = false;
    for (uint32_t count = 0; count < kMaxKicks && !done; count++) {
      if (cur < c) {  // bucket c lies past the table: never written here
        uint32_t* b = a.slots + static_cast<uint64_t>(cur) * kB;
#pragma unroll
        for (int j = 0; j < kB; j++) {
          if (!done && b[j] == 0u && atomicCAS(b + j, 0u, tag) == 0u) done = true;
        }
        if (!done && count > 0) {
          const uint32_t r = kick_rand(rng) % kB;
          const uint32_t old = atomicExch(b + r, tag);
          if (old == 0u) {
            done = true;
          } else {
            tag = old;
          }
        }
      }
      if (!done) cur = cuckoo_alt(cur, tag, a.addr);
    }
    if (!done) {
      // victim cache (cuckoofilter_logic.hpp:318-320); when it is taken the
      // tag in hand is lost, the reference's `insert == false`.
      uint32_t* v = a.table + a.victim_word;
      if (atomicCAS(v + 2, 0u, 1u) == 0u) {
        v[0] = cur;
        v[1] = tag;
      } else {
        atomicAdd(a.failed, 1ull);
      }
    }
  }
}

// Packs the slot array back into the reference's byte layout, one 32-bit
// output word per thread; bits outside tags keep their old value.
template <class Cfg>
__global__ void cuckoo_pack_kernel(uint32_t* table, const uint32_t* slots, uint32_t bucket_cnt,
                                   uint64_t table_words) {
  constexpr int kT = Cfg::kT, kB = Cfg::kB, kBPB = Cfg::kBytesPerBucket;
  for (uint64_t w = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; w < table_words;
       w += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t b0 = (w * 4) / kBPB;
    uint64_t b1 = (w * 4 + 3) / kBPB;
    if (b1 >= bucket_cnt) b1 = bucket_cnt - 1;
    unsigned long long bits = 0, mask = 0;
    for (uint64_t bb = b0; bb <= b1; bb++) {
#pragma unroll
      for (int j = 0; j < kB; j++) {
        const int64_t rel = static_cast<int64_t>(bb * kBPB * 8 + static_cast<uint64_t>(kT) * j) -
                            static_cast<int64_t>(w * 32);
        const unsigned long long tv = slots[bb * kB + j] & Cfg::kTagMask;
        const unsigned long long tm = Cfg::kTagMask;
        if (rel >= 32 || rel <= -kT) continue;
        if (rel >= 0) {
          bits |= tv << rel;
          mask |= tm << rel;
        } else {
          bits |= tv >> (-rel);
          mask |= tm >> (-rel);
        }
      }
    }
    const uint32_t m32 = static_cast<uint32_t>(mask);
    table[w] = (table[w] & ~m32) | (static_cast<uint32_t>(bits) & m32);
  }
}

template <class Cfg>
__global__ void cuckoo_count_kernel(const uint32_t* table, uint32_t bucket_cnt, uint64_t victim_word,
                                    unsigned long long* count) {
  unsigned long long c = 0;
  const uint64_t n = static_cast<uint64_t>(bucket_cnt) * Cfg::kB;
  for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < n;
       s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    c += CuckooOps<Cfg>::read_tag(table, s / Cfg::kB, static_cast<int>(s % Cfg::kB)) != 0u;
  }
  for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(0xffffffffu, c, d);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
  if (blockIdx.x == 0 && threadIdx.x == 0 && (table[victim_word + 2] & 0xffu)) atomicAdd(count, 1ull);
}

#endif  // __CUDACC__

}  // namespace dtlg
