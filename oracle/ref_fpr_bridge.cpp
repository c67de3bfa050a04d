// ref_fpr_bridge.cpp -- C ABI over the reference's analytic false-positive
// rate formulas, compiled from its own headers (TEST INFRASTRUCTURE ONLY).
//
//   dtl::bloomfilter::fpr(m, n, k, B, S, z, self_collisions)  fpr.hpp:12-51
//   dtl::bloomfilter::fpr(m, n, config)                       fpr.hpp:54-61
//   dtl::cuckoofilter::fpr(associativity, tag_bits, load)     math.hpp:199-205
//
// Boost's Poisson pmf comes from ref_shim/boost/math/distributions/poisson.hpp.
#include <cstdint>
#include <stdexcept>

#include <dtl/dtl.hpp>
#include <dtl/filter/blocked_bloomfilter/blocked_bloomfilter_config.hpp>
#include <dtl/filter/blocked_bloomfilter/fpr.hpp>

extern "C" {

// The reference's fpr(m, n, config) (self collisions on, its default);
// returns -1 when it throws.
double ref_bbf_fpr(uint64_t m, uint64_t n, uint32_t k, uint32_t word_size, uint32_t w, uint32_t s,
                   uint32_t z) {
  try {
    dtl::blocked_bloomfilter_config c;
    c.k = k;
    c.word_size = word_size;
    c.word_cnt_per_block = w;
    c.sector_cnt = s;
    c.zone_cnt = z;
    return dtl::bloomfilter::fpr(m, n, c);
  } catch (...) {
    return -1.0;
  }
}

double ref_cf_fpr(uint32_t tags_per_bucket, uint32_t bits_per_tag, double load_factor) {
  return dtl::cuckoofilter::fpr(tags_per_bucket, bits_per_tag, load_factor);
}

}  // extern "C"
