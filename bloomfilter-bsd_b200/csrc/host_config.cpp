// host_config.cpp -- see host_config.hpp.
#include "host_config.hpp"

#include <algorithm>

namespace dtlg {

namespace {
bool is_pow2(uint64_t x) { return x == 1 || (x && !(x & (x - 1))); }  // math.hpp:13-15
uint64_t next_pow2(uint64_t v) { return v <= 1 ? 1 : 1ull << (64 - __builtin_clzll(v - 1)); }
uint32_t ilog2(uint64_t v) { return 63u - static_cast<uint32_t>(__builtin_clzll(v)); }
}  // namespace

bool next_cheap_magic(uint32_t n, uint32_t* divisor, uint32_t* magic, uint32_t* shift) {
  const uint64_t d_max = 0xFFFFFFFFull - 2;  // div.hpp:18
  for (uint64_t d = std::max<uint32_t>(n, 2u); d <= d_max; ++d) {
    if ((d & (d - 1)) == 0) continue;
    const uint32_t L = ilog2(d);
    const unsigned __int128 num = static_cast<unsigned __int128>(1) << (32 + L);
    const uint64_t q = static_cast<uint64_t>(num / d);
    const uint64_t r = static_cast<uint64_t>(num % d);
    if (d - r >= (1ull << L)) continue;
    *divisor = static_cast<uint32_t>(d);
    *magic = static_cast<uint32_t>(q + 1);
    *shift = L;
    return true;
  }
  return false;
}

int make_addr(uint64_t desired, bool magic_mode, Addr* a) {
  const uint64_t max_blocks = 1ull << 31;  // block_addressing_logic.hpp:47,150
  *a = Addr{};
  if (desired > max_blocks) return 2;
  if (!magic_mode) {
    const uint64_t bc = next_pow2(desired);
    if (bc < desired || next_pow2(bc) > max_blocks) return 2;
    a->magic_mode = 0;
    a->block_cnt = static_cast<uint32_t>(bc);
    a->pow2_mul = static_cast<uint32_t>(bc);  // 2^log2(bc)
    a->block_cnt_mask = static_cast<uint32_t>(bc - 1);
  } else {
    uint32_t d, mg, sh;
    if (!next_cheap_magic(static_cast<uint32_t>(desired), &d, &mg, &sh)) return 2;
    if (d < desired || next_pow2(d) > max_blocks) return 2;
    a->magic_mode = 1;
    a->block_cnt = d;
    a->divisor = d;
    a->magic = mg;
    a->shift = sh;
    a->block_cnt_mask = static_cast<uint32_t>(next_pow2(d) - 1);
  }
  return 0;
}

int describe_bloom(uint32_t word_size, uint32_t w, uint32_t s, uint32_t z, uint32_t k, uint64_t m,
                   FilterDesc* d) {
  *d = FilterDesc{};
  auto one_of = [](uint32_t x, std::initializer_list<uint32_t> l) {
    return std::find(l.begin(), l.end(), x) != l.end();
  };
  if (word_size != 4 && word_size != 8) return 1;  // filter.hpp:64
  if (z == 1) {
    // blocked_bloomfilter.hpp:106-115,169-229
    if (!one_of(w, {1, 2, 4, 8, 16}) || !one_of(s, {1, 2, 4, 8, 16}) || k < 1 || k > 16) return 1;
    const uint32_t s_eff = std::min(w * word_size, s);
    const uint32_t k_eff = std::max(k % s_eff == 0 ? k : 1u, s_eff);
    if (s_eff != s || k_eff != k) return 1;
    d->kind = Kind::kBloom;
  } else {
    // zoned_blocked_bloomfilter.hpp:102-105,114-120,174-215
    if (w <= z || !one_of(w, {4, 8, 16}) || !one_of(z, {2, 4, 8})) return 1;
    if (k < 2 || k > 16 || (k & 1)) return 1;
    const uint32_t z_eff = std::min(w / 2, z);
    const uint32_t k_eff = std::max(k % z_eff == 0 ? k : 2u, z_eff);
    if (k_eff != k || z_eff != z) return 1;
    s = w;
    d->kind = Kind::kZoned;
  }
  d->word_bytes = word_size;
  d->w = w;
  d->s = s;
  d->z = z;
  d->k = k;
  d->m = m;
  const uint64_t block_bits = static_cast<uint64_t>(w) * word_size * 8;
  // blocked_bloomfilter.hpp:234-242; blocked_bloomfilter_logic.hpp:81-82
  const int rc = make_addr((m + block_bits - 1) / block_bits, !is_pow2(m), &d->addr);
  if (rc) return rc;
  d->m_actual = static_cast<uint64_t>(d->addr.block_cnt) * block_bits;
  d->word_cnt = static_cast<uint64_t>(d->addr.block_cnt) * w;
  // the reference forms word indexes in 32 bits (blocked_bloomfilter_logic.hpp:99)
  if (d->word_cnt > (1ull << 32)) return 2;
  d->size_u64 = word_size == 4 ? (d->word_cnt + 1) / 2 : d->word_cnt;  // bbf_32.cpp:80-82
  d->alloc_u64 = d->size_u64;  // the facade's allocation (filter.hpp:113-119)
  return 0;
}

int describe_cuckoo(uint32_t t, uint32_t b, uint64_t m, FilterDesc* d) {
  *d = FilterDesc{};
  // cuckoofilter.hpp:184-206
  if (!(t == 4 || t == 8 || t == 12 || t == 16 || t == 32)) return 1;
  if (!(b == 1 || b == 2 || b == 4)) return 1;
  d->kind = Kind::kCuckoo;
  d->t = t;
  d->b = b;
  d->m = m;
  d->bytes_per_bucket = (t * b + 7) / 8;  // cuckoofilter_table.hpp:89
  const uint64_t bucket_bits = d->bytes_per_bucket * 8ull;
  const int rc = make_addr((m + bucket_bits - 1) / bucket_bits, !is_pow2(m), &d->addr);
  if (rc) return rc;
  const uint64_t bytes = static_cast<uint64_t>(d->bytes_per_bucket) * d->addr.block_cnt;
  d->m_actual = bytes * 8;                  // cuckoofilter.hpp:259
  d->word_cnt = (bytes + 3) / 4;            // cuckoofilter_table.hpp:247-249
  d->victim_word = d->word_cnt;             // cuckoofilter_logic.hpp:157
  d->size_u64 = (d->word_cnt + 1) / 2;      // cf.cpp:77-79
  // table + 12-byte victim record + 32 bytes of slack for reads of bucket
  // index block_cnt, rounded to 16 bytes
  d->alloc_u64 = ((d->word_cnt * 4 + 12 + 32 + 15) / 16) * 2;
  return 0;
}

int describe_bcf(uint32_t block_bytes, uint32_t t, uint32_t a, uint64_t m, FilterDesc* d) {
  *d = FilterDesc{};
  // blocked_cuckoofilter.hpp:254-297
  if (!(block_bytes == 8 || block_bytes == 32 || block_bytes == 64 || block_bytes == 128 || block_bytes == 256 ||
        block_bytes == 512))
    return 1;
  if (!((t == 8 && a == 4) || (t == 8 && a == 8) || (t == 10 && a == 6) || (t == 12 && a == 4) ||
        (t == 16 && a == 2) || (t == 16 && a == 4)))
    return 1;
  d->kind = Kind::kBlockedCuckoo;
  d->t = t;
  d->b = a;
  d->m = m;
  d->block_bytes = block_bytes;
  d->word_bytes = t * a <= 32 ? 4 : 8;  // one bucket per word (blocked_cuckoofilter_logic.hpp:280-414)
  d->w = block_bytes / d->word_bytes;
  d->bucket_bits = ilog2(d->w);
  const uint64_t block_bits = block_bytes * 8ull;
  // blocked_cuckoofilter.hpp:303-312, blocked_cuckoofilter_logic.hpp:59-61
  const bool magic = !is_pow2(m);
  const int rc = make_addr((m + block_bits - 1) / block_bits, magic, &d->addr);
  if (rc) return rc;
  d->m_actual = static_cast<uint64_t>(d->addr.block_cnt) * block_bits;  // logic.hpp:262-264
  d->word_cnt = static_cast<uint64_t>(d->addr.block_cnt) * d->w;
  // the reference forms word indexes in 32 bits (blocked_cuckoofilter_logic.hpp:76)
  if (d->word_cnt > (1ull << 32)) return 2;
  // bucket hash: the block hash shifted past the addressing bits when enough
  // bits remain, else a second hash of the key (logic.hpp:77-82,
  // block_addressing_logic.hpp:131,230)
  const uint32_t req = magic ? 32u : ilog2(d->addr.block_cnt);
  d->hash_shift = req + t + d->bucket_bits <= 32 ? req : 32u;
  d->size_u64 = d->m_actual / 64;  // block_bytes >= 8: whole 64-bit words
  d->alloc_u64 = d->size_u64;
  return 0;
}

int describe_classic(uint32_t k, uint64_t m, bool magic, FilterDesc* d) {
  *d = FilterDesc{};
  // dyn::mul32 throws for hash numbers above 16 (hash_family.hpp:295-297),
  // from inside the reference's noexcept insert / contains: k <= 17
  if (k > 17) return 1;
  d->kind = Kind::kClassicBloom;
  d->k = k;
  d->m = m;
  d->word_bytes = 4;
  d->w = 1;
  const int rc = make_addr((m + 31) / 32, magic, &d->addr);  // bloomfilter_logic.hpp:62-64
  if (rc) return rc;
  d->word_cnt = d->addr.block_cnt;                  // :84-87
  d->m_actual = static_cast<uint64_t>(d->addr.block_cnt) * 32;  // :74-77
  // bit index (h >> (27 - addressing bits)) & 31 (:105,138), as the reference
  // compiles: a POW2 shift count taken mod 32, the MAGIC bit index 0
  if (magic) {
    d->bit_shift = 0;
    d->bit_mask = 0;
  } else {
    d->bit_shift = (27u - ilog2(d->addr.block_cnt)) & 31u;
    d->bit_mask = 31;
  }
  d->size_u64 = (d->word_cnt + 1) / 2;
  d->alloc_u64 = d->size_u64;
  return 0;
}

std::string filter_name(const FilterDesc& d) {
  const std::string addr = d.addr.magic_mode ? "\"magic\"" : "\"pow2\"";
  const uint64_t bytes = (d.m_actual + 7) / 8;
  if (d.kind == Kind::kClassicBloom) {
    // the reference's bloomfilter_logic has no name(): the blocked filters' format
    return "{\"name\":\"bloom\",\"size\":" + std::to_string(bytes) + ",\"k\":" + std::to_string(d.k) +
           ",\"addr\":" + addr + "}";
  }
  if (d.kind == Kind::kBlockedCuckoo) {
    // blocked_cuckoofilter.hpp:445-454
    return "{\"name\":\"blocked_cuckoo\", \"size\":" + std::to_string(bytes) +
           ",\"block_size\":" + std::to_string(d.block_bytes) + ",\"tag_bits\":" + std::to_string(d.t) +
           ",\"associativity\":" + std::to_string(d.b) + ",\"addr\":" + addr + "}";
  }
  if (d.kind == Kind::kCuckoo) {
    // cuckoofilter.hpp:335-342 ("u" is the SIMD unroll factor of the reference's
    // CPU path; the GPU has none, reported as 0)
    return "{\"name\":\"cuckoo\",\"size\":" + std::to_string(bytes) +
           ",\"tag_bits\":" + std::to_string(d.t) + ",\"associativity\":" + std::to_string(d.b) +
           ",\"delete_support\":false,\"u\":0,\"addr\":" + addr + "}";
  }
  // blocked_bloomfilter.hpp:381-389, zoned_blocked_bloomfilter.hpp:368-377
  std::string s = "{\"name\":\"blocked_bloom_multiword\",\"size\":" + std::to_string(bytes) +
                  ",\"word_size\":" + std::to_string(d.word_bytes) + ",\"k\":" + std::to_string(d.k) +
                  ",\"w\":" + std::to_string(d.w) + ",\"s\":" + std::to_string(d.s);
  if (d.kind == Kind::kZoned) s += ",\"z\":" + std::to_string(d.z);
  s += ",\"u\":0,\"e\":0,\"addr\":" + addr + "}";
  return s;
}

}  // namespace dtlg
