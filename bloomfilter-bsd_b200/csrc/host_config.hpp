// host_config.hpp -- filter construction rules on the host (validation, sizes,
// addressing, name).  Reference: blocked_bloomfilter.hpp:96-390,
// zoned_blocked_bloomfilter.hpp:98-378, cuckoofilter.hpp:115-343,
// blocked_cuckoofilter.hpp:183-455, bloomfilter_logic.hpp:59-87,
// block_addressing_logic.hpp:41-235, div.hpp:30-57, filter.hpp:42-72.
#pragma once

#include <cstdint>
#include <string>

#include "common.cuh"

namespace dtlg {

enum class Kind : int { kBloom = 0, kZoned = 1, kCuckoo = 2, kBlockedCuckoo = 3, kClassicBloom = 4 };

// Smallest d >= max(n, 2) whose libdivide u32 magic needs neither the add step
// nor the power-of-two shift path (div.hpp:30-57; libdivide.h:719-769, the
// round-up method: L = floor(log2 d), q = floor(2^(32+L) / d), cheap iff
// d - (2^(32+L) mod d) < 2^L, magic = q + 1, shift = L).
bool next_cheap_magic(uint32_t n, uint32_t* divisor, uint32_t* magic, uint32_t* shift);

// Returns 0 on success, 2 on a size error (the reference's logic_error).
int make_addr(uint64_t desired_blocks, bool magic_mode, Addr* out);

struct FilterDesc {
  Kind kind = Kind::kBloom;
  // Bloom
  uint32_t word_bytes = 4, w = 1, s = 1, z = 1, k = 8;
  // cuckoo (b = tags per bucket) and blocked cuckoo (b = associativity)
  uint32_t t = 16, b = 4, bytes_per_bucket = 8;
  // blocked cuckoo: block size, log2(buckets per block), bucket-hash shift
  // (32: the bucket hash is key * C[0]); word_bytes / w hold the bucket word
  // size and the buckets per block
  uint32_t block_bytes = 0, bucket_bits = 0, hash_shift = 32;
  // classic Bloom: bit index = (h >> bit_shift) & bit_mask (k above)
  uint32_t bit_shift = 0, bit_mask = 0;
  uint64_t m = 0, m_actual = 0;
  Addr addr{};
  uint64_t word_cnt = 0;      // Bloom: words of word_bytes; cuckoo: 32-bit table words
  uint64_t size_u64 = 0;      // filter_base::size()
  uint64_t alloc_u64 = 0;     // words the caller allocates
  uint64_t victim_word = 0;   // cuckoo: 32-bit word index of the victim record
};

// 0 ok, 1 invalid config, 2 size error.
int describe_bloom(uint32_t word_size, uint32_t w, uint32_t s, uint32_t z, uint32_t k, uint64_t m,
                   FilterDesc* out);
int describe_cuckoo(uint32_t t, uint32_t b, uint64_t m, FilterDesc* out);
int describe_bcf(uint32_t block_bytes, uint32_t t, uint32_t a, uint64_t m, FilterDesc* out);
int describe_classic(uint32_t k, uint64_t m, bool magic, FilterDesc* out);
std::string filter_name(const FilterDesc& d);

}  // namespace dtlg
