// bloom.cuh -- blocked Bloom filter probe / build for one compile-time config.
//
// Reference: blocked_bloomfilter_logic.hpp:95-136 (h0 = hash_0(key) selects
// the block; the block type sets / tests k bits) with the block types of
// blocked_bloomfilter_block_logic_{sgew,sltw,zoned}.hpp.  The bit layout comes
// from make_schedule() (common.cuh) and is identical to the reference's scalar
// insert / contains, so filters built here are byte-identical to CPU builds.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "probe.cuh"
#include "probe3.cuh"

namespace dtlg {

template <typename Word, int W, int S, int Z, int K>
struct BloomCfg {
  using word_t = Word;
  static constexpr int kW = W, kS = S, kZ = Z, kK = K;
  static constexpr int kBlockBytes = W * static_cast<int>(sizeof(Word));
  static constexpr Schedule sched =
      make_schedule(static_cast<uint32_t>(sizeof(Word) * 8), W, S, Z, K, /*stale_k8=*/true);
  static_assert(sched.ok, "config needs a hash function beyond the family");
};

struct BuildArgs {
  void* filter;
  const uint32_t* keys_al;
  uint64_t n_phys;
  uint32_t pre;
  Addr addr;
};

#ifdef __CUDACC__

template <typename Word>
__device__ __forceinline__ void atomic_or_word(Word* p, Word m) {
  if constexpr (sizeof(Word) == 8) {
    atomicOr(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(m));
  } else {
    atomicOr(reinterpret_cast<unsigned int*>(p), static_cast<unsigned int>(m));
  }
}

// 256-bit load (sm_100): 32 bytes from a 32-byte aligned address.
__device__ __forceinline__ void ld_nc_256(const void* p, unsigned long long& a, unsigned long long& b,
                                          unsigned long long& c, unsigned long long& d) {
  asm volatile("ld.global.nc.v4.u64 {%0,%1,%2,%3}, [%4];"
               : "=l"(a), "=l"(b), "=l"(c), "=l"(d)
               : "l"(p));
}

// The same without allocating the line in L1: for random blocks of a filter
// that does not fit L1 the allocation only costs L1TEX work (see ProbeArgs::l1na).
__device__ __forceinline__ void ld_nc_na_256(const void* p, unsigned long long& a, unsigned long long& b,
                                             unsigned long long& c, unsigned long long& d) {
  asm volatile("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
               : "=l"(a), "=l"(b), "=l"(c), "=l"(d)
               : "l"(p));
}

// Coherent (weak, L1-cacheable) loads for filter words written earlier in the
// same kernel (the batched build+probe kernel); the .nc path above may only
// read data that is constant for the whole kernel.
__device__ __forceinline__ uint4 ld_weak_128(const void* p) {
  uint4 r;
  asm volatile("ld.global.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w) : "l"(p));
  return r;
}
// 256 bits coherently, for a 32-byte aligned address: one L1 wavefront for a
// 32-byte half block where two 128-bit loads take two.
__device__ __forceinline__ void ld_weak_256(const void* p, unsigned long long& a, unsigned long long& b,
                                            unsigned long long& c, unsigned long long& d) {
  asm volatile("ld.global.v4.u64 {%0,%1,%2,%3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
}
__device__ __forceinline__ unsigned long long ld_weak_64(const void* p) {
  unsigned long long r;
  asm volatile("ld.global.u64 %0, [%1];" : "=l"(r) : "l"(p));
  return r;
}
__device__ __forceinline__ unsigned int ld_weak_32(const void* p) {
  unsigned int r;
  asm volatile("ld.global.u32 %0, [%1];" : "=r"(r) : "l"(p));
  return r;
}

// Loads a whole block of W words with the widest aligned vector loads.  Each
// load of a random block is one L1 wavefront, so fewer, wider loads raise the
// probe rate: blocks of >= 32 bytes use 256-bit loads when the filter base is
// 32-byte aligned (vec32), 128-bit loads otherwise; l1na = the 256-bit loads
// do not allocate in L1.  NC = false reads through the coherent path (see
// ld_weak_128).
template <typename Word, int W, bool NC = true>
__device__ __forceinline__ void load_block(const Word* base, Word (&v)[W], bool vec32 = false, bool l1na = false) {
  constexpr int kBytes = W * static_cast<int>(sizeof(Word));
  if constexpr (!NC) {
    if constexpr (kBytes >= 32) {
      if (vec32) {
        unsigned long long* d = reinterpret_cast<unsigned long long*>(&v[0]);
        const unsigned long long* p = reinterpret_cast<const unsigned long long*>(base);
#pragma unroll
        for (int i = 0; i < kBytes / 32; i++) ld_weak_256(p + 4 * i, d[4 * i], d[4 * i + 1], d[4 * i + 2], d[4 * i + 3]);
        return;
      }
    }
    if constexpr (kBytes >= 16) {
#pragma unroll
      for (int i = 0; i < kBytes / 16; i++) {
        const uint4 x = ld_weak_128(reinterpret_cast<const uint4*>(base) + i);
        uint32_t* d = reinterpret_cast<uint32_t*>(&v[0]) + 4 * i;
        d[0] = x.x; d[1] = x.y; d[2] = x.z; d[3] = x.w;
      }
    } else if constexpr (kBytes == 8) {
      *reinterpret_cast<unsigned long long*>(&v[0]) = ld_weak_64(base);
    } else {
      v[0] = static_cast<Word>(ld_weak_32(base));
    }
    return;
  }
  if constexpr (kBytes >= 32) {
    if (vec32) {
      unsigned long long* d = reinterpret_cast<unsigned long long*>(&v[0]);
      const unsigned long long* p = reinterpret_cast<const unsigned long long*>(base);
      if (l1na) {
#pragma unroll
        for (int i = 0; i < kBytes / 32; i++)
          ld_nc_na_256(p + 4 * i, d[4 * i], d[4 * i + 1], d[4 * i + 2], d[4 * i + 3]);
      } else {
#pragma unroll
        for (int i = 0; i < kBytes / 32; i++) ld_nc_256(p + 4 * i, d[4 * i], d[4 * i + 1], d[4 * i + 2], d[4 * i + 3]);
      }
      return;
    }
  }
  if constexpr (kBytes >= 16) {
    const uint4* p = reinterpret_cast<const uint4*>(base);
#pragma unroll
    for (int i = 0; i < kBytes / 16; i++) {
      const uint4 x = __ldg(p + i);
      uint32_t* d = reinterpret_cast<uint32_t*>(&v[0]) + 4 * i;
      d[0] = x.x; d[1] = x.y; d[2] = x.z; d[3] = x.w;
    }
  } else if constexpr (kBytes == 8) {
    const unsigned long long x = __ldg(reinterpret_cast<const unsigned long long*>(base));
    *reinterpret_cast<unsigned long long*>(&v[0]) = x;
  } else {
    v[0] = static_cast<Word>(__ldg(reinterpret_cast<const unsigned int*>(base)));
  }
}

// Groups of schedule `s` whose word lies in 32-byte chunk c of the block
// (chunk_words words per chunk).
constexpr int chunk_groups(const Schedule& s, int chunk_words, int c) {
  int n = 0;
  for (uint32_t g = 0; g < s.ng; g++)
    if (static_cast<int>(s.g[g].wconst) / chunk_words == c) n++;
  return n;
}

// True for hashed-word layouts (zoned, s < w) of 64-byte blocks in which
// every group picks its word from two neighbours within one 32-byte chunk,
// the groups in chunk order, and some chunk holds two or more groups (see
// BloomOps::kChunked).
constexpr bool chunked_layout(const Schedule& s, int w, int word_bytes) {
  const int bytes = w * word_bytes, cw = 32 / word_bytes;
  if (s.fixed_words || bytes != 64) return false;
  int prev = 0, most = 0;
  for (uint32_t g = 0; g < s.ng; g++) {
    const int lo = s.g[g].wconst, hi = lo + (1 << s.g[g].wbits) - 1;
    if (s.g[g].wbits > 1 || lo / cw != hi / cw || lo / cw < prev) return false;
    prev = lo / cw;
  }
  for (int c = 0; c < bytes / 32; c++) most = chunk_groups(s, cw, c) > most ? chunk_groups(s, cw, c) : most;
  return most >= 2;  // with one group per chunk the per-group loads are as few
}

template <class Cfg>
struct BloomOps {
  using Word = typename Cfg::word_t;
  static constexpr Schedule kS = Cfg::sched;
  static constexpr int kW = Cfg::kW;

  template <int G>
  __device__ __forceinline__ static Word group_mask(uint32_t key) {
    constexpr Group g = kS.g[G];
    Word m = 0;
    static_for<g.nbit>([&](auto J) {
      constexpr BitDraw b = g.bit[decltype(J)::value];
      const uint32_t v = (hash_sel<b.sel>(key) >> b.shift) & ((1u << b.bits) - 1u);
      m |= Word(1) << (v + b.off);
    });
    return m;
  }

  template <int G>
  __device__ __forceinline__ static uint32_t group_word(uint32_t key) {
    constexpr Group g = kS.g[G];
    if constexpr (g.wbits == 0) {
      return g.wconst;
    } else {
      return g.wconst + ((hash_sel<g.wsel>(key) >> g.wshift) & ((1u << g.wbits) - 1u));
    }
  }

  __device__ __forceinline__ static const Word* block_ptr(const void* filter, uint32_t key, const Addr& a) {
    const uint32_t blk = block_index(key * mul_const(0), a);
    return static_cast<const Word*>(filter) + static_cast<uint64_t>(blk) * kW;
  }

  // Every bit of the key set?  ((word & mask) == mask over all touched words.
  // The reference configures no early out, blocked_bloomfilter.hpp:34; the
  // result of the conjunction is the same with one, see kHalves.)
  __device__ __forceinline__ static bool contains(const ProbeArgs& a, uint32_t key) {
    const uint32_t blk = block_index(key * mul_const(0), a.addr);
    if (a.range_on && (blk < a.blk_lo || blk >= a.blk_hi)) return false;  // another pass's block
    return test_block<true>(static_cast<const Word*>(a.filter) + static_cast<uint64_t>(blk) * kW, key,
                            a.vec32 != 0, a.l1na != 0);
  }

  // The groups whose word lies in [Lo, Hi), against words v[0..Hi-Lo).
  template <int Lo, int Hi>
  __device__ __forceinline__ static bool test_words(const Word* v, uint32_t key) {
    bool ok = true;
    static_for<kS.ng>([&](auto G) {
      constexpr int g = decltype(G)::value;
      constexpr int wi = kS.g[g].wconst;
      if constexpr (wi >= Lo && wi < Hi) {
        const Word m = group_mask<g>(key);
        ok &= (v[wi - Lo] & m) == m;
      }
    });
    return ok;
  }

  // Groups [Lo, Hi) of a layout whose words the hash picks: one word load each.
  template <int Lo, int Hi, bool NC = true>
  __device__ __forceinline__ static bool test_groups(const Word* base, uint32_t key) {
    bool ok = true;
    static_for<kS.ng>([&](auto G) {
      constexpr int g = decltype(G)::value;
      if constexpr (g >= Lo && g < Hi) {
        const Word m = group_mask<g>(key);
        const Word* p = base + group_word<g>(key);
        Word x;
        if constexpr (sizeof(Word) == 8) {
          x = NC ? __ldg(reinterpret_cast<const unsigned long long*>(p)) : ld_weak_64(p);
        } else {
          x = NC ? __ldg(reinterpret_cast<const unsigned int*>(p)) : ld_weak_32(p);
        }
        ok &= (x & m) == m;
      }
    });
    return ok;
  }

  // Blocks of >= 64 bytes test their first half before loading the second:
  // the match result is the same (the test is a conjunction), but most
  // non-members fail on the first half, so the second 32-byte load is skipped
  // for them.
  static constexpr bool kHalves = kS.fixed_words && kW * static_cast<int>(sizeof(Word)) >= 64;

  // Layouts whose words the hash picks (zoned, s < w) in 64-byte blocks,
  // where each group picks one of two neighbouring words of a 32-byte chunk
  // known at compile time (zones and sectors of 16 bytes: u64 w=8 z=4 or
  // s=4, u32 w=16 z=8 or s=8): the chunk is read with one 256-bit load and
  // each group's word is picked from it in registers, instead of one load per
  // group.  Random loads cost the L1 about one wavefront per cache line and
  // instruction, whatever their width, so these layouts need half the load
  // instructions or fewer.  The groups of chunk 0 come first (zones and
  // sectors are drawn in block order); they are tested before chunk 1 is
  // loaded.  Measured on B200 (2^28 probes, 10 % hits, 8 MiB / 256 MiB,
  // Gkeys/s, per-group loads -> chunks): u64 w=8 z=4 k=8 162.8 -> 170.9 /
  // 91.4 -> 108.1; u64 w=8 s=4 k=8 91.4 -> 152.4 / 76.2 -> 74.3; u32 w=16 s=8
  // k=8 101.8 -> 203.7 / 80.3 -> 88.8.  Wider picks (four or eight words:
  // u64 s=2, u32 s=2, u32 z=4), 32-byte blocks and more than 8 bits per key
  // hold more registers, spill in the 32-register kernels and were slower or
  // no faster (u64 w=8 s=2 k=8 at 256 MiB 78.6 -> 47.1), so they keep the
  // per-group loads.
  static constexpr int kChunkWords = 32 / static_cast<int>(sizeof(Word));
  static constexpr bool kChunked = chunked_layout(kS, kW, static_cast<int>(sizeof(Word))) && Cfg::kK <= 8;
  static constexpr int kChunk0 = chunk_groups(kS, kChunkWords, 0);  // groups tested against chunk 0

  // Group G's word, picked from the words c[] of its chunk.
  template <int G>
  __device__ __forceinline__ static Word chunk_word(const Word (&c)[kChunkWords], uint32_t key) {
    constexpr Group g = kS.g[G];
    constexpr int lo = g.wconst % kChunkWords;
    Word x = c[lo];
    if constexpr (g.wbits > 0) {
      const uint32_t j = (hash_sel<g.wsel>(key) >> g.wshift) & ((1u << g.wbits) - 1u);
      static_for<(1 << g.wbits) - 1>([&](auto J) {
        constexpr int jj = decltype(J)::value + 1;
        if (j == jj) x = c[lo + jj];
      });
    }
    return x;
  }

  // Groups [Lo, Hi) against the words of their chunk.
  template <int Lo, int Hi>
  __device__ __forceinline__ static bool test_chunk(const Word (&c)[kChunkWords], uint32_t key) {
    bool ok = true;
    static_for<kS.ng>([&](auto G) {
      constexpr int g = decltype(G)::value;
      if constexpr (g >= Lo && g < Hi) {
        const Word m = group_mask<g>(key);
        ok &= (chunk_word<g>(c, key) & m) == m;
      }
    });
    return ok;
  }

  // The key's bits in the block at `base`; NC selects the read-only load path.
  template <bool NC>
  __device__ __forceinline__ static bool test_block(const Word* base, uint32_t key, bool vec32, bool l1na = false) {
    if constexpr (kChunked) {
      if (vec32) {
        Word c[kChunkWords];
        load_block<Word, kChunkWords, NC>(base, c, true, l1na);
        if (!test_chunk<0, kChunk0>(c, key)) return false;
        if constexpr (kChunk0 < static_cast<int>(kS.ng)) {
          load_block<Word, kChunkWords, NC>(base + kChunkWords, c, true, l1na);
          return test_chunk<kChunk0, kS.ng>(c, key);
        } else {
          return true;
        }
      }
    }
    if constexpr (kHalves) {
      constexpr int kH = kW / 2;
      if constexpr (NC) {
        if (vec32) {
          Word v[kH];
          load_block<Word, kH>(base, v, true, l1na);
          if (!test_words<0, kH>(v, key)) return false;
          load_block<Word, kH>(base + kH, v, true, l1na);
          return test_words<kH, kW>(v, key);
        }
      } else {
        Word v[kH];
        load_block<Word, kH, false>(base, v, vec32);
        if (!test_words<0, kH>(v, key)) return false;
        load_block<Word, kH, false>(base + kH, v, vec32);
        return test_words<kH, kW>(v, key);
      }
    }
    bool ok = true;
    if constexpr (kS.fixed_words) {
      Word v[kW];
      load_block<Word, kW, NC>(base, v, vec32, l1na);
      static_for<kS.ng>([&](auto G) {
        constexpr int g = decltype(G)::value;
        const Word m = group_mask<g>(key);
        ok &= (v[kS.g[g].wconst] & m) == m;
      });
    } else if constexpr (kS.ng >= 2) {
      // words picked by the hash (zoned, s < w): the first half of the groups,
      // then, for the keys that pass, the second half
      constexpr int kG = kS.ng / 2;
      if (!test_groups<0, kG, NC>(base, key)) return false;
      return test_groups<kG, kS.ng, NC>(base, key);
    } else {
      ok = test_groups<0, kS.ng, NC>(base, key);
    }
    return ok;
  }

  // test_block<NC> for N keys at once: the N first halves (or first groups)
  // are loaded before any of them is tested, then the second halves of the
  // keys that passed, so a thread has N gathers in flight instead of one (for
  // kernels that run at half the SM's warp slots).  Only the keys whose bit is
  // set in `live` are loaded and tested.  Bit q of the result: key q matches.
  // (In the 64-register bitmask kernel, at the same half occupancy, four keys
  // per thread this way made L2-resident probes slower: 8 MiB u64 w=8 s=8 k=8,
  // 182 -> 151 Gkeys/s.)
  template <int N, bool NC>
  __device__ __forceinline__ static uint32_t testn(const Word* const* base, const uint32_t* key, uint32_t live,
                                                   bool vec32, bool l1na = false) {
    uint32_t hit = 0;
    auto one_by_one = [&]() {
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((live >> q) & 1u) hit |= (test_block<NC>(base[q], key[q], vec32, l1na) ? 1u : 0u) << q;
    };
    if constexpr (kChunked) {
      if (vec32) {
        Word c[N][kChunkWords];
#pragma unroll
        for (int q = 0; q < N; q++)
          if ((live >> q) & 1u) load_block<Word, kChunkWords, NC>(base[q], c[q], true, l1na);
        uint32_t pass = 0;
#pragma unroll
        for (int q = 0; q < N; q++)
          if ((live >> q) & 1u) pass |= (test_chunk<0, kChunk0>(c[q], key[q]) ? 1u : 0u) << q;
        if constexpr (kChunk0 == static_cast<int>(kS.ng)) {
          return pass;
        } else {
#pragma unroll
          for (int q = 0; q < N; q++)
            if ((pass >> q) & 1u) load_block<Word, kChunkWords, NC>(base[q] + kChunkWords, c[q], true, l1na);
#pragma unroll
          for (int q = 0; q < N; q++)
            if ((pass >> q) & 1u) hit |= (test_chunk<kChunk0, kS.ng>(c[q], key[q]) ? 1u : 0u) << q;
          return hit;
        }
      }
    }
    if constexpr (kHalves) {
      if (NC && !vec32) {  // the read-only path tests halves only with 256-bit loads
        one_by_one();
        return hit;
      }
      constexpr int kH = kW / 2;
      Word v[N][kH];
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((live >> q) & 1u) load_block<Word, kH, NC>(base[q], v[q], vec32, l1na);
      uint32_t pass = 0;
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((live >> q) & 1u) pass |= (test_words<0, kH>(v[q], key[q]) ? 1u : 0u) << q;
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((pass >> q) & 1u) load_block<Word, kH, NC>(base[q] + kH, v[q], vec32, l1na);
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((pass >> q) & 1u) hit |= (test_words<kH, kW>(v[q], key[q]) ? 1u : 0u) << q;
    } else if constexpr (!kS.fixed_words && kS.ng >= 2) {
      constexpr int kG = kS.ng / 2;
      constexpr int kSlots = kG > kS.ng - kG ? kG : kS.ng - kG;  // words held per key and phase
      Word x[N][kSlots];
      auto load_groups = [&](auto lo_c, auto hi_c, int q) {
        constexpr int Lo = decltype(lo_c)::value, Hi = decltype(hi_c)::value;
        static_for<kS.ng>([&](auto G) {
          constexpr int g = decltype(G)::value;
          if constexpr (g >= Lo && g < Hi) {
            const Word* p = base[q] + group_word<g>(key[q]);
            if constexpr (sizeof(Word) == 8) {
              x[q][g - Lo] = NC ? __ldg(reinterpret_cast<const unsigned long long*>(p)) : ld_weak_64(p);
            } else {
              x[q][g - Lo] = static_cast<Word>(NC ? __ldg(reinterpret_cast<const unsigned int*>(p)) : ld_weak_32(p));
            }
          }
        });
      };
      auto test_loaded = [&](auto lo_c, auto hi_c, int q) {
        constexpr int Lo = decltype(lo_c)::value, Hi = decltype(hi_c)::value;
        bool ok = true;
        static_for<kS.ng>([&](auto G) {
          constexpr int g = decltype(G)::value;
          if constexpr (g >= Lo && g < Hi) {
            const Word m = group_mask<g>(key[q]);
            ok &= (x[q][g - Lo] & m) == m;
          }
        });
        return ok;
      };
      using C0 = std::integral_constant<int, 0>;
      using CG = std::integral_constant<int, kG>;
      using CN = std::integral_constant<int, kS.ng>;
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((live >> q) & 1u) load_groups(C0{}, CG{}, q);
      uint32_t pass = 0;
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((live >> q) & 1u) pass |= (test_loaded(C0{}, CG{}, q) ? 1u : 0u) << q;
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((pass >> q) & 1u) load_groups(CG{}, CN{}, q);
#pragma unroll
      for (int q = 0; q < N; q++)
        if ((pass >> q) & 1u) hit |= (test_loaded(CG{}, CN{}, q) ? 1u : 0u) << q;
    } else {
      one_by_one();
    }
    return hit;
  }

  // The same test against a copy of the filter in shared memory (plan 4):
  // plain loads, which the compiler issues as shared-memory loads.
  __device__ __forceinline__ static bool contains_shared(const void* sfilter, const ProbeArgs& a, uint32_t key) {
    const uint32_t blk = block_index(key * mul_const(0), a.addr);
    const Word* base = static_cast<const Word*>(sfilter) + static_cast<uint64_t>(blk) * kW;
    constexpr int kBytes = kW * static_cast<int>(sizeof(Word));
    bool ok = true;
    if constexpr (kS.fixed_words) {
      Word v[kW];
      if constexpr (kBytes >= 16) {
#pragma unroll
        for (int i = 0; i < kBytes / 16; i++) {
          const uint4 x = reinterpret_cast<const uint4*>(base)[i];
          uint32_t* d = reinterpret_cast<uint32_t*>(&v[0]) + 4 * i;
          d[0] = x.x; d[1] = x.y; d[2] = x.z; d[3] = x.w;
        }
      } else {
#pragma unroll
        for (int i = 0; i < kW; i++) v[i] = base[i];
      }
      static_for<kS.ng>([&](auto G) {
        constexpr int g = decltype(G)::value;
        const Word m = group_mask<g>(key);
        ok &= (v[kS.g[g].wconst] & m) == m;
      });
    } else {
      static_for<kS.ng>([&](auto G) {
        constexpr int g = decltype(G)::value;
        const Word m = group_mask<g>(key);
        ok &= (base[group_word<g>(key)] & m) == m;
      });
    }
    return ok;
  }

  __device__ __forceinline__ static void insert(void* filter, uint32_t key, const Addr& a) {
    Word* base = const_cast<Word*>(block_ptr(filter, key, a));
    static_for<kS.ng>([&](auto G) {
      constexpr int g = decltype(G)::value;
      atomic_or_word<Word>(base + group_word<g>(key), group_mask<g>(key));
    });
  }

  // Warp-cooperative insert.  Every lane brings one key (valid or not); the
  // kS.ng word updates of each key are spread over kS.ng lanes, so one warp
  // instruction carries the updates of 32 / kS.ng whole keys and those of one
  // key reach the L2 in one request per 32-byte sector, where they are applied
  // together.  One thread per key issues its kS.ng atomic ORs one after the
  // other, each a request of its own: on B200, 64-byte blocks of 8 u64 words
  // with one bit each, 2^26 keys into 8 MiB build at 82.6 Gkeys/s this way
  // against 23.6 (and into 512 MiB at 24.5 against 6.7).  All 32 lanes call it.
  static constexpr bool kLaneInsert = kS.ng >= 2 && kS.ng <= 32 && (32 % kS.ng) == 0;
  // Per warp, in shared memory.  Entry (key lane l, group g) sits at
  // g * 32 + (l ^ (g * 32 / kS.ng)): a lane's stores of one group are 32
  // consecutive entries, and the loads of a round, kS.ng groups of each of
  // 32 / kS.ng keys, fall in distinct banks (a [key][group] layout made every
  // store a 16-way bank conflict for 8 u64 groups).
  struct LaneStage {
    Word mask[32 * kS.ng];
    uint8_t word[32 * kS.ng];   // word of the group in its block (hashed layouts)
    uint32_t blk[32];           // block of each lane's key
  };
  __device__ __forceinline__ static void insert_lanes(void* filter, uint32_t key, bool valid, const Addr& a,
                                                      LaneStage& st) {
    static_assert(kLaneInsert, "groups per key must divide the warp");
    constexpr int kNg = kS.ng;
    constexpr uint32_t kPer = 32 / kNg;  // keys per round
    const uint32_t lane = threadIdx.x & 31u;
    st.blk[lane] = block_index(key * mul_const(0), a);
    static_for<kNg>([&](auto G) {
      constexpr int g = decltype(G)::value;
      const uint32_t e = g * 32 + (lane ^ (g * kPer));
      st.mask[e] = valid ? group_mask<g>(key) : Word(0);
      if constexpr (!kS.fixed_words) st.word[e] = static_cast<uint8_t>(group_word<g>(key));
    });
    // with fixed words, this lane's group (lane % kNg) always has the same word
    uint32_t wl = 0;
    if constexpr (kS.fixed_words) {
      static_for<kNg>([&](auto G) {
        constexpr int g = decltype(G)::value;
        if (lane % kNg == g) wl = kS.g[g].wconst;
      });
    }
    __syncwarp();
    const uint32_t g = lane % kNg;  // this lane's group in every round
#pragma unroll
    for (int j = 0; j < kNg; j++) {
      const uint32_t kl = j * kPer + lane / kNg;  // lane of the key
      const uint32_t e = g * 32 + (kl ^ (g * kPer));
      const Word m = st.mask[e];
      const uint32_t w = kS.fixed_words ? wl : st.word[e];
      if (m) atomic_or_word<Word>(static_cast<Word*>(filter) + static_cast<uint64_t>(st.blk[kl]) * kW + w, m);
    }
    __syncwarp();
  }
};

// batch_insert (blocked_bloomfilter_logic.hpp:111-117).  The reference inserts
// sequentially with a CAS-OR per word (..._sgew.hpp:300-325); OR commutes, so
// concurrent atomic ORs give the same words in any order.
// Layouts with 2..32 word groups per key insert warp-cooperatively
// (BloomOps::insert_lanes); the loop then runs warp-uniformly.
template <class Cfg>
__global__ void __launch_bounds__(256) bloom_build_kernel(const __grid_constant__ BuildArgs a) {
  using Ops = BloomOps<Cfg>;
  const uint4* keys4 = reinterpret_cast<const uint4*>(a.keys_al);
  const uint64_t nvec = (a.n_phys + 3) >> 2;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  if constexpr (Ops::kLaneInsert) {
    __shared__ typename Ops::LaneStage st[8];
    typename Ops::LaneStage& my = st[threadIdx.x >> 5];
    for (uint64_t vb = blockIdx.x * static_cast<uint64_t>(blockDim.x) + (threadIdx.x & ~31u); vb < nvec;
         vb += stride) {
      const uint64_t v = vb + (threadIdx.x & 31u);
      const uint4 kv = v < nvec ? __ldcs(keys4 + v) : make_uint4(0, 0, 0, 0);
      const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint64_t p = v * 4 + q;
        Ops::insert_lanes(a.filter, k[q], p >= a.pre && p < a.n_phys, a.addr, my);
      }
    }
  } else {
    for (uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; v < nvec; v += stride) {
      const uint4 kv = __ldcs(keys4 + v);
      const uint32_t k[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint64_t p = v * 4 + q;
        if (p >= a.pre && p < a.n_phys) Ops::insert(a.filter, k[q], a.addr);
      }
    }
  }
}

// batch_insert of range-grouped (key, position) pairs (probe3.cuh's
// partition): consecutive keys hit the same L2-sized block range, so the
// atomic ORs of a filter far larger than L2 update lines that sit in L2.  Keys
// whose run overflowed its segment are inserted from the key array (inserting
// a key twice sets the same bits).
template <class Cfg>
__global__ void __launch_bounds__(256) bloom_build_pairs_kernel(const __grid_constant__ PartArgs pa, void* filter,
                                                                const Addr addr) {
  using Ops = BloomOps<Cfg>;
  auto ins = [&](uint32_t key, uint32_t) { Ops::insert(filter, key, addr); };
  if constexpr (Ops::kLaneInsert) {
    __shared__ typename Ops::LaneStage st[8];
    typename Ops::LaneStage& my = st[threadIdx.x >> 5];
    for_each_pair_warp(seg_chunks(pa), [&](uint32_t key, bool valid) { Ops::insert_lanes(filter, key, valid, addr, my); });
  } else {
    for_each_pair(seg_chunks(pa), ins);
  }
  for_each_overflow_key(pa, ins);
}

#endif  // __CUDACC__

}  // namespace dtlg
