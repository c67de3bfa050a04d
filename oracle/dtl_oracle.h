/*
 * dtl_oracle.h -- CPU restatement of the DTL filter build/probe path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load
 * it.  The product library (libdtlg.so) never links or calls it.
 *
 * It restates, in plain C, the reference algorithm of peterboncz/bloomfilter-bsd
 * ("dtl"): multiplicative hashing, POW2/MAGIC block addressing, the blocked
 * Bloom filter bit layouts (sgew / sltw / zoned) and the partial-key cuckoo
 * filter.  Each function cites the reference file:line it follows.  The
 * restatement is pinned against the reference's own known-answer test
 * (src/dtl/filter/filter_test.cpp:16-40) and against the reference compiled
 * from its sources (oracle/_ref, see oracle/Makefile) over a config sweep.
 */
#ifndef DTL_ORACLE_H
#define DTL_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_OK = 0, ORC_ERR_CONFIG = 1, ORC_ERR_SIZE = 2 };
enum { ORC_ADDR_POW2 = 0, ORC_ADDR_MAGIC = 1 };

/* key * C[idx] mod 2^32 (hash_family.hpp:20-122). idx in [0,16]. */
uint32_t orc_hash(uint32_t key, uint32_t idx);

/* next_cheap_magic (div.hpp:30-57): smallest d >= max(n,2) whose libdivide
 * u32 magic needs neither the add step nor the shift path. Returns 0 if none. */
int orc_next_cheap_magic(uint32_t n, uint32_t *divisor, uint32_t *magic, uint32_t *shift);

/* fast_mod_u32 (div.hpp:88-92). */
uint32_t orc_fast_mod(uint32_t a, uint32_t divisor, uint32_t magic, uint32_t shift);

/* Block addressing (block_addressing_logic.hpp:41-235). */
typedef struct {
  uint32_t mode;        /* ORC_ADDR_POW2 or ORC_ADDR_MAGIC */
  uint32_t block_cnt;
  uint32_t block_cnt_log2;  /* log2(next_pow2(block_cnt)) */
  uint32_t block_cnt_mask;  /* next_pow2(block_cnt) - 1 */
  uint32_t magic, shift;    /* MAGIC only */
} orc_addr;

int orc_addr_init(orc_addr *a, uint64_t desired_block_cnt, uint32_t mode);
uint32_t orc_addr_block(const orc_addr *a, uint32_t hash_value);

/* ---------------------------------------------------------------------------
 * Blocked Bloom filter (blocked_bloomfilter.hpp, zoned_blocked_bloomfilter.hpp,
 * blocked_bloomfilter_logic.hpp).
 * ------------------------------------------------------------------------- */
typedef struct {
  uint32_t word_bytes;  /* 4 or 8 */
  uint32_t w, s, z, k;  /* words/block, sectors, zones (1 = not zoned), bits/key */
  orc_addr addr;
  uint64_t m;           /* desired bits */
  uint64_t m_actual;    /* block_cnt * block bits */
  uint64_t word_cnt;    /* words of word_bytes */
  uint64_t size_u64;    /* filter_base::size(): 64-bit words the facade allocates */
} orc_bloom;

/* Validates like the runtime dispatchers (blocked_bloomfilter.hpp:96-116,
 * 169-229; zoned_blocked_bloomfilter.hpp:98-215) and sizes the filter. */
int orc_bloom_init(orc_bloom *f, uint32_t word_bytes, uint32_t w, uint32_t s,
                   uint32_t z, uint32_t k, uint64_t m);

/* stale_k8 = 1 reproduces the reference's scalar path (insert / contains),
 * whose unrolled k=8 word block does not hand its hash value on
 * (blocked_bloomfilter_block_logic_sgew_specialization.hpp:69-167);
 * stale_k8 = 0 is the reference's SIMD contains path. */
void orc_bloom_insert(const orc_bloom *f, void *data, const uint32_t *keys,
                      uint64_t n, int stale_k8);
int orc_bloom_contains(const orc_bloom *f, const void *data, uint32_t key, int stale_k8);
uint64_t orc_bloom_batch_contains(const orc_bloom *f, const void *data,
                                  const uint32_t *keys, uint32_t n,
                                  uint32_t *match_pos, uint32_t match_offset,
                                  int stale_k8);
/* In-block (word index, bit index) pairs of one key, k entries each. */
void orc_bloom_bits(const orc_bloom *f, uint32_t key, int stale_k8,
                    uint32_t *word_idx, uint32_t *bit_idx);

/* ---------------------------------------------------------------------------
 * Cuckoo filter (cuckoofilter.hpp, cuckoofilter_logic.hpp, cuckoofilter_table.hpp)
 * ------------------------------------------------------------------------- */
typedef struct {
  uint32_t t, b;            /* bits per tag, tags per bucket */
  uint32_t bytes_per_bucket;
  orc_addr addr;
  uint64_t m, m_actual;
  uint64_t table_words_u32; /* victim cache lives at this 32-bit word */
  uint64_t size_u64;        /* cf::size() of the reference (excludes the victim cache) */
  uint64_t alloc_u64;       /* words to allocate: table + victim cache + read slack */
} orc_cuckoo;

int orc_cuckoo_init(orc_cuckoo *f, uint32_t t, uint32_t b, uint64_t m);
/* Sequential insert (cuckoofilter_logic.hpp:292-337); kick slots from a
 * seeded xorshift generator in place of the reference's thread-local mt19937.
 * Returns 1 when every key went in (the reference's batch_insert result). */
int orc_cuckoo_insert(const orc_cuckoo *f, void *data, const uint32_t *keys,
                      uint64_t n, uint64_t seed);
int orc_cuckoo_contains(const orc_cuckoo *f, const void *data, uint32_t key);
uint64_t orc_cuckoo_batch_contains(const orc_cuckoo *f, const void *data,
                                   const uint32_t *keys, uint32_t n,
                                   uint32_t *match_pos, uint32_t match_offset);
uint64_t orc_cuckoo_count_occupied(const orc_cuckoo *f, const void *data);
uint32_t orc_cuckoo_read_tag(const orc_cuckoo *f, const void *data, uint64_t i, uint32_t j);
void orc_cuckoo_index_tag(const orc_cuckoo *f, uint32_t key, uint32_t *i1, uint32_t *i2, uint32_t *tag);

/* ---------------------------------------------------------------------------
 * Blocked cuckoo filter (blocked_cuckoofilter/blocked_cuckoofilter*.hpp,
 * wrapped as dtl::bcf in bcf.hpp:11-63).  Each block is a small cuckoo table
 * of one-word buckets; a key touches only its own block.
 * ------------------------------------------------------------------------- */
typedef struct {
  uint32_t block_bytes;     /* 8, 32, 64, 128, 256 or 512 */
  uint32_t t, a;            /* bits per tag, tags per bucket (associativity) */
  uint32_t word_bytes;      /* one bucket = one word: 4 if t*a <= 32, else 8 */
  uint32_t bucket_bits;     /* log2(buckets per block) */
  uint32_t hash_shift;      /* POW2 with log2(B) + t + bucket_bits <= 32: log2(B)
                               (bucket hash = block hash << log2(B)); else 32:
                               the bucket hash is key * C[0] */
  orc_addr addr;
  uint64_t m, m_actual;
  uint64_t word_cnt;        /* words of word_bytes */
  uint64_t size_u32;        /* blocked_cuckoofilter::size(): 32-bit words */
} orc_bcf;

int orc_bcf_init(orc_bcf *f, uint32_t block_bytes, uint32_t t, uint32_t a, uint64_t m);
/* Sequential insert (blocked_cuckoofilter_logic.hpp:73-95); kick slots from a
 * seeded xorshift generator in place of the reference's thread-local mt19937. */
void orc_bcf_insert(const orc_bcf *f, void *data, const uint32_t *keys, uint64_t n, uint64_t seed);
int orc_bcf_contains(const orc_bcf *f, const void *data, uint32_t key);
uint64_t orc_bcf_batch_contains(const orc_bcf *f, const void *data, const uint32_t *keys,
                                uint32_t n, uint32_t *match_pos, uint32_t match_offset);
/* Block, both bucket indexes and the tag of a key. */
void orc_bcf_locate(const orc_bcf *f, uint32_t key, uint32_t *block, uint32_t *b1, uint32_t *b2,
                    uint32_t *tag);

/* ---------------------------------------------------------------------------
 * Classic Bloom filter (bloomfilter/bloomfilter_logic.hpp:22-212): one bit in
 * each of k independently addressed 32-bit words.
 * ------------------------------------------------------------------------- */
typedef struct {
  uint32_t k;               /* bits per key, 0..17 (hash functions C[0..k-1]) */
  orc_addr addr;            /* one "block" per 32-bit word */
  uint32_t bit_shift;       /* bit index = (h >> bit_shift) & bit_mask */
  uint32_t bit_mask;
  uint64_t m, m_actual;
  uint64_t word_cnt;        /* bloomfilter_logic::size(): 32-bit words */
} orc_cbf;

/* mode: ORC_ADDR_POW2 or ORC_ADDR_MAGIC (the reference's template argument). */
int orc_cbf_init(orc_cbf *f, uint32_t k, uint64_t m, uint32_t mode);
void orc_cbf_insert(const orc_cbf *f, void *data, const uint32_t *keys, uint64_t n);
int orc_cbf_contains(const orc_cbf *f, const void *data, uint32_t key);
uint64_t orc_cbf_batch_contains(const orc_cbf *f, const void *data, const uint32_t *keys,
                                uint32_t n, uint32_t *match_pos, uint32_t match_offset);

/* Parallel (pthreads) batch_contains over contiguous slices; used only as the
 * timed CPU baseline.  Returns the total match count; per-slice positions are
 * written to match_pos[slice_begin ...] (not compacted). */
uint64_t orc_bloom_batch_contains_mt(const orc_bloom *f, const void *data,
                                     const uint32_t *keys, uint64_t n,
                                     uint32_t *match_pos, int threads);

#ifdef __cplusplus
}
#endif
#endif
