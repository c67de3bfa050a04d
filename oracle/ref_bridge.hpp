// ref_bridge.hpp -- C entry points over the reference's OWN filter logic.
//
// TEST INFRASTRUCTURE ONLY.  This file holds no reference code: it includes the
// reference headers from their place in the reference tree (the include path is
// set by oracle/Makefile) and instantiates the logic types directly, the way
// the reference's runtime dispatchers do (blocked_bloomfilter.hpp:49-54,
// zoned_blocked_bloomfilter.hpp:49-56, cuckoofilter.hpp:56-68).  The built
// library (oracle/_ref/libdtlref_*.so) pins the C restatement in
// oracle/dtl_oracle.c and serves as the timed CPU baseline.
#pragma once

#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include <dtl/dtl.hpp>
#include <dtl/simd.hpp>
#include <dtl/simd/extensions.hpp>
#include <dtl/filter/blocked_bloomfilter/hash_family.hpp>
#include <dtl/filter/blocked_bloomfilter/block_addressing_logic.hpp>
#include <dtl/filter/blocked_bloomfilter/blocked_bloomfilter_logic.hpp>
#include <dtl/filter/blocked_bloomfilter/blocked_bloomfilter_block_logic.hpp>
#include <dtl/filter/blocked_bloomfilter/blocked_bloomfilter_block_logic_zoned.hpp>
#include <dtl/filter/cuckoofilter/cuckoofilter_logic.hpp>

namespace refbridge {

using key_t = uint32_t;
using hash_value_t = uint32_t;
constexpr uint64_t kLanes = dtl::simd::lane_count<uint32_t>;

// Type-erased operations of one instantiated filter logic.
struct ops {
  void* (*create)(uint64_t m);
  void (*destroy)(void*);
  uint64_t (*word_cnt)(void*);
  uint64_t (*length)(void*);
  int (*insert)(void*, void* data, const uint32_t* keys, uint32_t n);
  int (*contains)(void*, const void* data, uint32_t key);
  uint64_t (*batch_contains)(void*, const void* data, const uint32_t* keys, uint32_t n,
                             uint32_t* out, uint32_t off, int unroll);
  uint64_t (*count_occupied)(void*, const void* data);
};

struct entry {
  uint32_t a, b, c, d, e, addr;  // bloom: word bytes, w, s, z, k ; cuckoo: t, b, 0, 0, 0
  const ops* o;
};

void register_bloom(const entry& e);
void register_cuckoo(const entry& e);

// blocked_bloomfilter<Tw>::bbf (blocked_bloomfilter.hpp:49-54)
template <typename Tw, uint32_t W, uint32_t S, uint32_t K, dtl::block_addressing A>
using bbf_logic = dtl::blocked_bloomfilter_logic<
    key_t, dtl::hasher,
    typename dtl::blocked_bloomfilter_block_logic<key_t, Tw, W, S, K, dtl::hasher, hash_value_t,
                                                  false, 1>::type,
    A, false>;

// zoned_blocked_bloomfilter<Tw>::bbf (zoned_blocked_bloomfilter.hpp:49-56)
template <typename Tw, uint32_t W, uint32_t Z, uint32_t K, dtl::block_addressing A>
using zbbf_logic = dtl::blocked_bloomfilter_logic<
    key_t, dtl::hasher,
    dtl::multizone_block<key_t, Tw, W, Z, K, dtl::hasher, hash_value_t, 1, 0, Z, false>, A,
    false>;

// cuckoofilter::cf (cuckoofilter.hpp:60-68)
template <uint32_t T, uint32_t B, dtl::block_addressing A>
using cf_logic = dtl::cuckoofilter::cuckoofilter_logic<T, B, dtl::cuckoofilter::cuckoofilter_table, A>;

template <typename L>
struct bloom_ops {
  using word_t = typename L::word_t;
  static void* create(uint64_t m) { return new L(m); }
  static void destroy(void* p) { delete static_cast<L*>(p); }
  static uint64_t word_cnt(void* p) { return static_cast<L*>(p)->word_cnt(); }
  static uint64_t length(void* p) { return static_cast<L*>(p)->get_length(); }
  static int insert(void* p, void* data, const uint32_t* keys, uint32_t n) {
    static_cast<L*>(p)->batch_insert(static_cast<word_t*>(data), keys, n);
    return 1;
  }
  static int contains(void* p, const void* data, uint32_t key) {
    return static_cast<L*>(p)->contains(static_cast<const word_t*>(data), key) ? 1 : 0;
  }
  static uint64_t batch_contains(void* p, const void* data, const uint32_t* keys, uint32_t n,
                                 uint32_t* out, uint32_t off, int unroll) {
    const L* l = static_cast<L*>(p);
    const word_t* d = static_cast<const word_t*>(data);
    switch (unroll) {
      case 0: return l->template batch_contains<0>(d, keys, n, out, off);
      case 2: return l->template batch_contains<kLanes * 2>(d, keys, n, out, off);
      case 4: return l->template batch_contains<kLanes * 4>(d, keys, n, out, off);
      default: return l->template batch_contains<kLanes>(d, keys, n, out, off);
    }
  }
  static uint64_t count_occupied(void*, const void*) { return 0; }
  static constexpr ops table = {create, destroy, word_cnt, length, insert,
                                contains, batch_contains, count_occupied};
};
template <typename L> constexpr ops bloom_ops<L>::table;

template <typename L>
struct cuckoo_ops {
  using word_t = typename L::word_t;
  static void* create(uint64_t m) { return new L(m); }
  static void destroy(void* p) { delete static_cast<L*>(p); }
  static uint64_t word_cnt(void* p) { return static_cast<L*>(p)->word_cnt(); }
  static uint64_t length(void* p) { return static_cast<L*>(p)->size_in_bytes() * 8; }
  static int insert(void* p, void* data, const uint32_t* keys, uint32_t n) {
    return static_cast<L*>(p)->batch_insert(static_cast<word_t*>(data), keys, n) ? 1 : 0;
  }
  static int contains(void* p, const void* data, uint32_t key) {
    return static_cast<L*>(p)->contains(static_cast<const word_t*>(data), key) ? 1 : 0;
  }
  static uint64_t batch_contains(void* p, const void* data, const uint32_t* keys, uint32_t n,
                                 uint32_t* out, uint32_t off, int unroll) {
    const L* l = static_cast<L*>(p);
    const word_t* d = static_cast<const word_t*>(data);
    // the unroll factors of the reference's cuckoo tuner, u in {0,1,2,4,8}
    // (cuckoofilter_tune_impl.hpp:50,149)
    switch (unroll) {
      case 0: return l->batch_contains_scalar(d, keys, n, out, off);
      case 2: return l->template batch_contains<kLanes * 2>(d, keys, n, out, off);
      case 4: return l->template batch_contains<kLanes * 4>(d, keys, n, out, off);
      case 8: return l->template batch_contains<kLanes * 8>(d, keys, n, out, off);
      default: return l->template batch_contains<kLanes>(d, keys, n, out, off);
    }
  }
  static uint64_t count_occupied(void* p, const void* data) {
    return static_cast<L*>(p)->count_occupied_slots(static_cast<const word_t*>(data));
  }
  static constexpr ops table = {create, destroy, word_cnt, length, insert,
                                contains, batch_contains, count_occupied};
};
template <typename L> constexpr ops cuckoo_ops<L>::table;

}  // namespace refbridge
