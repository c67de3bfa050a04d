// common.cuh -- shared device/host definitions of the dtlg kernels.
//
// The Bloom filter layouts of the reference (sgew, sltw, zoned) all reduce to
// "for each touched word: word index, bit mask", where every word index and bit
// index is a fixed slice of one of the family hashes key * C[i].  The slices
// depend only on the config, so they are computed here at COMPILE TIME into a
// `Schedule`; the kernels then unroll it and the compiler folds every shift and
// mask into constants.
#pragma once

#include <cstdint>
#include <utility>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace dtlg {

// hash_family.hpp:20-122: the multiplicative family, key * C[i] mod 2^32.
// C[0] addresses the block (bucket); the in-block draws start at C[1]
// (blocked_bloomfilter.hpp:46).
__host__ __device__ constexpr uint32_t mul_const(int i) {
  constexpr uint32_t c[17] = {
      596572387u,  370248451u,  2654435769u, 1799596469u, 0x9e3779b1u, 2284105051u,
      1203114875u, 1150766481u, 2729912477u, 1884591559u, 770785867u,  2667333959u,
      1550580529u, 0xcc9e2d51u, 0x1b873593u, 0x85ebca6bu, 0xc2b2ae35u};
  return c[i];
}

// Hash selector meaning "the constant 0": the reference's scalar draw chain
// starts from hash value 0 and, after its unrolled k=8 word block, keeps using
// the value it held before that block (see make_schedule).
constexpr uint8_t kSelZero = 255;

// One bit draw: value = (H[sel] >> shift) & (2^bits - 1), plus `off`.
struct BitDraw {
  uint8_t sel = 0, shift = 0, bits = 0, off = 0;
};

// One touched word: index = wconst + draw(wsel, wshift, wbits) (wbits = 0:
// a fixed word), and nbit bit draws whose bits are set / tested in that word.
struct Group {
  uint8_t wsel = 0, wshift = 0, wbits = 0, wconst = 0;
  uint8_t nbit = 0;
  BitDraw bit[16] = {};
};

struct Schedule {
  Group g[16] = {};
  uint32_t ng = 0;
  bool ok = true;         // false: the config would need a hash beyond C[16]
  bool fixed_words = true;  // every group has a fixed word (sgew)
};

// Running state of the top-down draw stream: the selector of the current hash
// value, the index of the next hash function, and the bits left in the value.
struct DrawStream {
  uint8_t sel = kSelZero, next = 1, rem = 0;
  bool ok = true;
  constexpr BitDraw take(uint32_t b) {
    if (rem < b) {  // rehash with the next function of the family
      if (next > 16) ok = false;
      sel = next;
      next = static_cast<uint8_t>(next + 1);
      rem = 32;
    }
    BitDraw d;
    d.sel = sel;
    d.shift = static_cast<uint8_t>(rem - b);
    d.bits = static_cast<uint8_t>(b);
    rem = static_cast<uint8_t>(rem - b);
    return d;
  }
};

constexpr uint32_t clog2(uint32_t x) { return x <= 1 ? 0 : 1 + clog2(x >> 1); }

// k_per bits into one word holding s_pw sectors (the reference's word_block,
// blocked_bloomfilter_block_logic_sgew.hpp:43-154).  Its unrolled k=8 twin
// (..._sgew_specialization.hpp:35-167), used by the scalar insert and contains,
// computes its eight draws but does not hand the hash value back, so the draws
// that follow continue from the value held before the block (index and bit
// count do advance).  `stale_k8` reproduces that.
constexpr void word_block(DrawStream& st, Group& g, uint32_t word_bits, uint32_t s_pw,
                          uint32_t k_per, bool stale_k8) {
  const uint32_t sector_bits = word_bits / s_pw;
  const uint32_t b = clog2(sector_bits);
  const uint32_t k_per_sector = k_per / s_pw;
  const uint8_t saved = st.sel;
  for (uint32_t j = 0; j < k_per; j++) {
    BitDraw d = st.take(b);
    d.off = static_cast<uint8_t>((j / k_per_sector) * sector_bits);
    g.bit[g.nbit++] = d;
  }
  if (stale_k8 && k_per == 8) st.sel = saved;
}

// The in-block layout of (word_bits, w words, s sectors, z zones, k bits):
//  * z > 1  : zoned (blocked_bloomfilter_block_logic_zoned.hpp:174-210)
//  * s >= w : sgew, word by word (..._sgew.hpp:347-376)
//  * s < w  : sltw, sector by sector (..._sltw.hpp:193-218, 504-528)
constexpr Schedule make_schedule(uint32_t word_bits, uint32_t w, uint32_t s, uint32_t z, uint32_t k,
                                 bool stale_k8) {
  Schedule sc;
  DrawStream st;
  const uint32_t lb = clog2(word_bits);
  if (z > 1) {
    const uint32_t wpz = w / z;
    for (uint32_t t = 0; t < z; t++) {
      Group& g = sc.g[sc.ng++];
      BitDraw wd = st.take(clog2(wpz));
      g.wsel = wd.sel;
      g.wshift = wd.shift;
      g.wbits = wd.bits;
      g.wconst = static_cast<uint8_t>(t * wpz);
      word_block(st, g, word_bits, 1, k / z, stale_k8);
    }
    sc.fixed_words = false;
  } else if (s >= w) {
    for (uint32_t i = 0; i < w; i++) {
      Group& g = sc.g[sc.ng++];
      g.wconst = static_cast<uint8_t>(i);
      word_block(st, g, word_bits, s / w, k / w, stale_k8);
    }
  } else {
    const uint32_t wps = w / s;
    const uint32_t lw = clog2(wps);
    for (uint32_t t = 0; t < s; t++) {
      for (uint32_t j = 0; j < k / s; j++) {
        // one draw of lw + lb bits: high lw bits pick the word in the sector,
        // low lb bits the bit in the word
        BitDraw d = st.take(lw + lb);
        Group& g = sc.g[sc.ng++];
        g.wsel = d.sel;
        g.wshift = static_cast<uint8_t>(d.shift + lb);
        g.wbits = static_cast<uint8_t>(lw);
        g.wconst = static_cast<uint8_t>(t * wps);
        BitDraw bd = d;
        bd.bits = static_cast<uint8_t>(lb);
        bd.off = 0;
        g.bit[g.nbit++] = bd;
      }
    }
    sc.fixed_words = false;
  }
  sc.ok = st.ok;
  return sc;
}

// ---- compile-time loops ------------------------------------------------------
template <class F, int... I>
__host__ __device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

template <int SEL>
__host__ __device__ __forceinline__ uint32_t hash_sel(uint32_t key) {
  if constexpr (SEL == kSelZero) {
    return 0u;
  } else {
    return key * mul_const(SEL);
  }
}

// ---- block (bucket) addressing: block_addressing_logic.hpp:104-110, 205-210 ----
struct Addr {
  uint32_t magic_mode;  // 0 = POW2, 1 = MAGIC
  uint32_t pow2_mul;    // POW2: 2^log2(block_cnt); h >> (32 - log2) == mulhi(h, 2^log2)
  uint32_t divisor;     // MAGIC: block count d and its cheap magic (div.hpp:88-92)
  uint32_t magic;
  uint32_t shift;
  uint32_t block_cnt;
  uint32_t block_cnt_mask;  // next_pow2(block_cnt) - 1 (cuckoo POW2 alt index)
};

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t block_index(uint32_t h, const Addr& a) {
  if (a.magic_mode) {
    const uint32_t q = __umulhi(h, a.magic) >> a.shift;
    return h - q * a.divisor;
  }
  // With a single POW2 block the reference shifts by 32 (undefined in C++);
  // mulhi(h, 1) == 0 defines it as block 0.
  return __umulhi(h, a.pow2_mul);
}

// block_index with the addressing mode fixed at compile time (no run-time
// branch on it; kernels bound by instruction issue instantiate both).
template <bool MAGIC>
__device__ __forceinline__ uint32_t block_index_of(uint32_t h, const Addr& a) {
  if constexpr (MAGIC) {
    const uint32_t q = __umulhi(h, a.magic) >> a.shift;
    return h - q * a.divisor;
  } else {
    return __umulhi(h, a.pow2_mul);
  }
}
#endif

}  // namespace dtlg
