/*
 * dtl_oracle.c -- CPU restatement of the DTL filter build/probe path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle the tests compare against, never the product): see dtl_oracle.h.
 *
 * Every function below restates the behaviour of the reference
 * (peterboncz/bloomfilter-bsd, paths relative to that project) in plain C.
 * The Bloom filter draws are simulated per key with an explicit
 * (hash value, hash index, remaining bits) state machine -- deliberately a
 * different formulation from the compile-time schedules of the CUDA kernels,
 * so that the two cross-check each other.
 */
#include "dtl_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* hash_family.hpp:20-122 -- the 17 multiplicative constants of mul32<.., i>. */
static const uint32_t kMul[17] = {
  596572387u,  370248451u,  2654435769u, 1799596469u, 0x9e3779b1u,
  2284105051u, 1203114875u, 1150766481u, 2729912477u, 1884591559u,
  770785867u,  2667333959u, 1550580529u, 0xcc9e2d51u, 0x1b873593u,
  0x85ebca6bu, 0xc2b2ae35u};

uint32_t orc_hash(uint32_t key, uint32_t idx) {
  if (idx > 16) abort();  /* the reference has no mul32<.., 17> */
  return key * kMul[idx];
}

static int is_pow2_u64(uint64_t x) {          /* math.hpp:13-15 */
  return x == 1 ? 1 : (x && ((x & (x - 1)) == 0));
}
static uint64_t next_pow2_u64(uint64_t v) {   /* math.hpp:17-19 (v >= 1) */
  if (v <= 1) return 1;
  return 1ull << (64 - __builtin_clzll(v - 1));
}
static uint32_t log2_u64(uint64_t v) { return 63u - (uint32_t)__builtin_clzll(v); }

/* div.hpp:30-57 over libdivide_u32_gen (thirdparty/libdivide/libdivide.h:719-769):
 * for d not a power of two, L = floor(log2 d), q = floor(2^(32+L)/d),
 * r = 2^(32+L) mod d; the "cheap" (no add marker) case is d - r < 2^L, with
 * magic q+1 and shift L.  This is the round-up method of Granlund/Montgomery
 * as implemented by libdivide's branchy generator. */
int orc_next_cheap_magic(uint32_t n, uint32_t *divisor, uint32_t *magic, uint32_t *shift) {
  const uint32_t d_max = 0xFFFFFFFFu - 2u;
  if (n < 2) n = 2;
  for (uint64_t d = n; d <= d_max; d++) {
    if ((d & (d - 1)) == 0) continue;                 /* shift path */
    uint32_t L = 31u - (uint32_t)__builtin_clz((uint32_t)d);
    uint64_t num = 1ull << (32 + L);
    uint64_t q = num / d, r = num % d;
    uint64_t e = d - r;
    if (e >= (1ull << L)) continue;                   /* needs the add step */
    *divisor = (uint32_t)d;
    *magic = (uint32_t)(q + 1);
    *shift = L;
    return 1;
  }
  return 0;
}

uint32_t orc_fast_mod(uint32_t a, uint32_t divisor, uint32_t magic, uint32_t shift) {
  uint32_t hi = (uint32_t)(((uint64_t)a * magic) >> 32);   /* div.hpp:69-72 */
  return a - (hi >> shift) * divisor;                       /* div.hpp:88-92 */
}

/* block_addressing_logic.hpp:61-83 (MAGIC) and :163-184 (POWER_OF_TWO). */
int orc_addr_init(orc_addr *a, uint64_t desired, uint32_t mode) {
  const uint64_t max_block_cnt = 1ull << 31;
  memset(a, 0, sizeof(*a));
  a->mode = mode;
  if (desired > max_block_cnt) return ORC_ERR_SIZE;
  if (mode == ORC_ADDR_POW2) {
    uint64_t bc = next_pow2_u64(desired);
    if (bc < desired || next_pow2_u64(bc) > max_block_cnt) return ORC_ERR_SIZE;
    a->block_cnt = (uint32_t)bc;
    a->block_cnt_log2 = log2_u64(bc);
    a->block_cnt_mask = (uint32_t)(bc - 1);
  } else {
    uint32_t d, mg, sh;
    if (!orc_next_cheap_magic((uint32_t)desired, &d, &mg, &sh)) return ORC_ERR_SIZE;
    if (d < desired || next_pow2_u64(d) > max_block_cnt) return ORC_ERR_SIZE;
    a->block_cnt = d;
    a->block_cnt_log2 = log2_u64(next_pow2_u64(d));
    a->block_cnt_mask = (uint32_t)(next_pow2_u64(d) - 1);
    a->magic = mg;
    a->shift = sh;
  }
  return ORC_OK;
}

/* get_block_idx: block_addressing_logic.hpp:104-110 and :205-210.  With a
 * single POW2 block the reference shifts a u32 by 32 (undefined in C++; its
 * SIMD path yields 0).  The restatement defines that case as block 0. */
uint32_t orc_addr_block(const orc_addr *a, uint32_t h) {
  if (a->mode == ORC_ADDR_POW2) {
    if (a->block_cnt_log2 == 0) return 0;
    return h >> (32u - a->block_cnt_log2);
  }
  return orc_fast_mod(h, a->block_cnt, a->magic, a->shift);
}

/* ======================================================================== */
/* Blocked Bloom filter                                                      */
/* ======================================================================== */

static uint32_t log2_u32(uint32_t x) { return 31u - (uint32_t)__builtin_clz(x); }
static uint32_t max_u32(uint32_t a, uint32_t b) { return a > b ? a : b; }
static uint32_t min_u32(uint32_t a, uint32_t b) { return a < b ? a : b; }

int orc_bloom_init(orc_bloom *f, uint32_t word_bytes, uint32_t w, uint32_t s,
                   uint32_t z, uint32_t k, uint64_t m) {
  memset(f, 0, sizeof(*f));
  /* filter.hpp:42-66: word size 4 or 8, zone_cnt == 1 selects bbf, else zbbf */
  if (word_bytes != 4 && word_bytes != 8) return ORC_ERR_CONFIG;
  if (z == 1) {
    /* blocked_bloomfilter.hpp:169-229: w,s in {1,2,4,8,16}; s clamped to
     * w*sizeof(word); k in 1..16 replaced by max(k%s==0 ? k : 1, s); the ctor
     * (:106-115) rejects the config when anything changed. */
    if (!(w == 1 || w == 2 || w == 4 || w == 8 || w == 16)) return ORC_ERR_CONFIG;
    if (!(s == 1 || s == 2 || s == 4 || s == 8 || s == 16)) return ORC_ERR_CONFIG;
    if (k < 1 || k > 16) return ORC_ERR_CONFIG;
    uint32_t s_eff = min_u32(w * word_bytes, s);
    uint32_t k_eff = max_u32((k % s_eff == 0) ? k : 1, s_eff);
    if (s_eff != s || k_eff != k) return ORC_ERR_CONFIG;
  } else {
    /* zoned_blocked_bloomfilter.hpp:102-105, 174-215 */
    if (w <= z) return ORC_ERR_CONFIG;
    if (!(w == 4 || w == 8 || w == 16)) return ORC_ERR_CONFIG;
    if (!(z == 2 || z == 4 || z == 8)) return ORC_ERR_CONFIG;
    if (k < 2 || k > 16 || (k & 1)) return ORC_ERR_CONFIG;
    uint32_t z_eff = min_u32(w / 2, z);
    uint32_t k_eff = max_u32((k % z_eff == 0) ? k : 2, z_eff);
    if (k_eff != k || z_eff != z) return ORC_ERR_CONFIG;
    s = w;
  }
  f->word_bytes = word_bytes; f->w = w; f->s = s; f->z = z; f->k = k; f->m = m;
  const uint64_t block_bits = (uint64_t)w * word_bytes * 8;
  /* blocked_bloomfilter.hpp:234-242: POW2 iff m is a power of two;
   * blocked_bloomfilter_logic.hpp:81-82: ceil(m / block bits) blocks */
  uint32_t mode = is_pow2_u64(m) ? ORC_ADDR_POW2 : ORC_ADDR_MAGIC;
  int rc = orc_addr_init(&f->addr, (m + block_bits - 1) / block_bits, mode);
  if (rc) return rc;
  f->m_actual = (uint64_t)f->addr.block_cnt * block_bits;   /* logic.hpp:181-183 */
  f->word_cnt = (uint64_t)f->addr.block_cnt * w;            /* logic.hpp:190-192 */
  /* The reference forms the word index in 32 bits (logic.hpp:99,130); beyond
   * 2^32 words it would wrap, so such sizes are rejected here. */
  if (f->word_cnt > (1ull << 32)) return ORC_ERR_SIZE;
  /* bbf_32.cpp:80-82 / bbf_64.cpp:81-83: size() in 64-bit words */
  f->size_u64 = word_bytes == 4 ? (f->word_cnt + 1) / 2 : f->word_cnt;
  return ORC_OK;
}

typedef struct {
  uint32_t key, hval, idx, rem;
} draw_state;

/* One draw of b bits, top down, re-hashing with the next function of the
 * family when fewer than b bits are left (the rehash rule of
 * blocked_bloomfilter_block_logic_sgew.hpp:68-82, ..._sltw.hpp:69-70,101-112,
 * ..._zoned.hpp:84-87,116-120). */
static uint32_t draw(draw_state *st, uint32_t b) {
  if (st->rem < b) {
    st->hval = orc_hash(st->key, st->idx);
    st->idx++;
    st->rem = 32;
  }
  uint32_t v = (st->hval >> (st->rem - b)) & ((1u << b) - 1u);
  st->rem -= b;
  return v;
}

/* word_block (sgew.hpp:43-154, k=8 twin sgew_specialization.hpp:35-230):
 * k_per bits in one word holding s_pw sectors; bit j lands in sector
 * j / (k_per / s_pw).  The k=8 twin (scalar) leaves the caller's hash value
 * untouched while the index and the remaining bit count advance. */
static void word_block(draw_state *st, uint32_t word_bits, uint32_t s_pw, uint32_t k_per,
                       uint32_t word, int stale_k8, uint32_t *wi, uint32_t *bi, uint32_t *n) {
  const uint32_t sector_bits = word_bits / s_pw;
  const uint32_t b = log2_u32(sector_bits);
  const uint32_t k_per_sector = k_per / s_pw;
  const uint32_t saved = st->hval;
  for (uint32_t j = 0; j < k_per; j++) {
    uint32_t v = draw(st, b);
    wi[*n] = word;
    bi[*n] = v + (j / k_per_sector) * sector_bits;
    (*n)++;
  }
  if (stale_k8 && k_per == 8) st->hval = saved;
}

void orc_bloom_bits(const orc_bloom *f, uint32_t key, int stale_k8,
                    uint32_t *wi, uint32_t *bi) {
  const uint32_t word_bits = f->word_bytes * 8;
  /* blocked_bloomfilter.hpp:46: the in-block draws start at hash function 1
   * with no bits left (the scalar entry points start from hash value 0). */
  draw_state st = {key, 0u, 1u, 0u};
  uint32_t n = 0;
  if (f->z > 1) {
    /* multizone_block (zoned.hpp:174-210): per zone one draw picks the word
     * inside the zone, then a word block of k/z bits in that word. */
    const uint32_t wpz = f->w / f->z;
    const uint32_t bz = log2_u32(wpz);
    for (uint32_t t = 0; t < f->z; t++) {
      uint32_t word = t * wpz + draw(&st, bz);
      word_block(&st, word_bits, 1, f->k / f->z, word, stale_k8, wi, bi, &n);
    }
  } else if (f->s >= f->w) {
    /* multiword_block (sgew.hpp:347-376): word by word, k/w bits each, the
     * word holding s/w sectors (type switch: block_logic.hpp:35). */
    for (uint32_t i = 0; i < f->w; i++)
      word_block(&st, word_bits, f->s / f->w, f->k / f->w, i, stale_k8, wi, bi, &n);
  } else {
    /* multisector_block / multiword_sector (sltw.hpp:193-218, 504-528): sector
     * by sector, each bit one draw of log2(w/s)+log2(word bits) bits whose
     * high part selects the word inside the sector. */
    const uint32_t wps = f->w / f->s;
    const uint32_t lw = log2_u32(wps), lb = log2_u32(word_bits);
    for (uint32_t t = 0; t < f->s; t++) {
      for (uint32_t j = 0; j < f->k / f->s; j++) {
        uint32_t x = draw(&st, lw + lb);
        wi[n] = t * wps + (x >> lb);
        bi[n] = x & (word_bits - 1u);
        n++;
      }
    }
  }
}

/* blocked_bloomfilter_logic.hpp:95-104 (insert) / :126-136 (contains):
 * h0 = hash_0(key) selects the block, whose first word is block * w. */
static uint64_t block_word0(const orc_bloom *f, uint32_t key) {
  uint32_t blk = orc_addr_block(&f->addr, orc_hash(key, 0));
  return (uint64_t)blk * f->w;
}

void orc_bloom_insert(const orc_bloom *f, void *data, const uint32_t *keys,
                      uint64_t n, int stale_k8) {
  uint32_t wi[16], bi[16];
  for (uint64_t i = 0; i < n; i++) {
    uint64_t base = block_word0(f, keys[i]);
    orc_bloom_bits(f, keys[i], stale_k8, wi, bi);
    for (uint32_t j = 0; j < f->k; j++) {
      if (f->word_bytes == 4) ((uint32_t *)data)[base + wi[j]] |= 1u << bi[j];
      else ((uint64_t *)data)[base + wi[j]] |= 1ull << bi[j];
    }
  }
}

int orc_bloom_contains(const orc_bloom *f, const void *data, uint32_t key, int stale_k8) {
  uint32_t wi[16], bi[16];
  uint64_t base = block_word0(f, key);
  orc_bloom_bits(f, key, stale_k8, wi, bi);
  /* (word & mask) == mask over every word (no early out,
   * blocked_bloomfilter.hpp:34) is the same as "every bit set". */
  for (uint32_t j = 0; j < f->k; j++) {
    uint64_t word = f->word_bytes == 4 ? ((const uint32_t *)data)[base + wi[j]]
                                       : ((const uint64_t *)data)[base + wi[j]];
    if (!((word >> bi[j]) & 1u)) return 0;
  }
  return 1;
}

/* blocked_bloomfilter_batch_dispatch.hpp:119-154: positions i + match_offset
 * (32-bit wrap) of the matching keys, ascending; returns the count. */
uint64_t orc_bloom_batch_contains(const orc_bloom *f, const void *data,
                                  const uint32_t *keys, uint32_t n,
                                  uint32_t *match_pos, uint32_t match_offset,
                                  int stale_k8) {
  uint64_t cnt = 0;
  for (uint32_t i = 0; i < n; i++)
    if (orc_bloom_contains(f, data, keys[i], stale_k8)) match_pos[cnt++] = i + match_offset;
  return cnt;
}

typedef struct {
  const orc_bloom *f;
  const void *data;
  const uint32_t *keys;
  uint64_t begin, end;
  uint32_t *out;
  uint64_t cnt;
} mt_arg;

static void *mt_worker(void *p) {
  mt_arg *a = (mt_arg *)p;
  a->cnt = orc_bloom_batch_contains(a->f, a->data, a->keys + a->begin,
                                    (uint32_t)(a->end - a->begin), a->out + a->begin,
                                    (uint32_t)a->begin, 1);
  return NULL;
}

uint64_t orc_bloom_batch_contains_mt(const orc_bloom *f, const void *data,
                                     const uint32_t *keys, uint64_t n,
                                     uint32_t *match_pos, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t th[256];
  mt_arg args[256];
  for (int t = 0; t < threads; t++) {
    args[t].f = f; args[t].data = data; args[t].keys = keys;
    args[t].begin = n * (uint64_t)t / (uint64_t)threads;
    args[t].end = n * (uint64_t)(t + 1) / (uint64_t)threads;
    args[t].out = match_pos; args[t].cnt = 0;
    pthread_create(&th[t], NULL, mt_worker, &args[t]);
  }
  uint64_t total = 0;
  for (int t = 0; t < threads; t++) { pthread_join(th[t], NULL); total += args[t].cnt; }
  return total;
}

/* ======================================================================== */
/* Cuckoo filter                                                             */
/* ======================================================================== */

#define ALT_MUL 0x5bd1e995u   /* cuckoofilter_logic.hpp:222,246 (MurmurHash2) */
#define MAX_KICKS 500u        /* cuckoofilter_logic.hpp:122 */

int orc_cuckoo_init(orc_cuckoo *f, uint32_t t, uint32_t b, uint64_t m) {
  memset(f, 0, sizeof(*f));
  /* cuckoofilter.hpp:184-206 */
  if (!(t == 4 || t == 8 || t == 12 || t == 16 || t == 32)) return ORC_ERR_CONFIG;
  if (!(b == 1 || b == 2 || b == 4)) return ORC_ERR_CONFIG;
  f->t = t; f->b = b; f->m = m;
  f->bytes_per_bucket = (t * b + 7) / 8;                 /* cuckoofilter_table.hpp:89 */
  const uint64_t bucket_bits = (uint64_t)f->bytes_per_bucket * 8;
  uint32_t mode = is_pow2_u64(m) ? ORC_ADDR_POW2 : ORC_ADDR_MAGIC;  /* cuckoofilter.hpp:211-213 */
  int rc = orc_addr_init(&f->addr, (m + bucket_bits - 1) / bucket_bits, mode);  /* logic.hpp:154-158 */
  if (rc) return rc;
  const uint64_t table_bytes = (uint64_t)f->bytes_per_bucket * f->addr.block_cnt;
  f->m_actual = table_bytes * 8;                         /* cuckoofilter.hpp:259 */
  f->table_words_u32 = (table_bytes + 3) / 4;            /* cuckoofilter_table.hpp:247-249 */
  f->size_u64 = (f->table_words_u32 + 1) / 2;            /* cf.cpp:77-79 */
  /* table, then the 12-byte victim record (logic.hpp:131-135,157), then slack
   * for reads of a bucket at index block_cnt (see cuckoo_alt below). */
  f->alloc_u64 = (f->table_words_u32 * 4 + 12 + 32 + 7) / 8;
  return ORC_OK;
}

static uint8_t *bucket_ptr(const orc_cuckoo *f, const void *data, uint64_t i) {
  return (uint8_t *)data + i * f->bytes_per_bucket;
}

/* cuckoofilter_table.hpp:111-136 (little endian) */
uint32_t orc_cuckoo_read_tag(const orc_cuckoo *f, const void *data, uint64_t i, uint32_t j) {
  const uint8_t *p = bucket_ptr(f, data, i);
  uint32_t tag = 0;
  uint16_t u16;
  switch (f->t) {
    case 4: tag = p[j >> 1] >> ((j & 1) << 2); break;
    case 8: tag = p[j]; break;
    case 12: memcpy(&u16, p + j + (j >> 1), 2); tag = (uint32_t)u16 >> ((j & 1) << 2); break;
    case 16: memcpy(&u16, p + 2 * j, 2); tag = u16; break;
    case 32: memcpy(&tag, p + 4 * j, 4); break;
  }
  return f->t == 32 ? tag : (tag & ((1u << f->t) - 1u));
}

/* cuckoofilter_table.hpp:143-178 */
static void write_tag(const orc_cuckoo *f, void *data, uint64_t i, uint32_t j, uint32_t tag) {
  uint8_t *p = bucket_ptr(f, data, i);
  uint16_t u16;
  if (f->t != 32) tag &= (1u << f->t) - 1u;
  switch (f->t) {
    case 4:
      p += j >> 1;
      if ((j & 1) == 0) *p = (uint8_t)((*p & 0xf0) | tag);
      else *p = (uint8_t)((*p & 0x0f) | (tag << 4));
      break;
    case 8: p[j] = (uint8_t)tag; break;
    case 12:
      p += j + (j >> 1);
      memcpy(&u16, p, 2);
      if ((j & 1) == 0) u16 = (uint16_t)((u16 & 0xf000) | tag);
      else u16 = (uint16_t)((u16 & 0x000f) | (tag << 4));
      memcpy(p, &u16, 2);
      break;
    case 16: u16 = (uint16_t)tag; memcpy(p + 2 * j, &u16, 2); break;
    case 32: memcpy(p + 4 * j, &tag, 4); break;
  }
}

/* cuckoofilter_logic.hpp:214-252.  The MAGIC form returns block_cnt (one past
 * the last bucket) when i == 0 and tag*M mod c == 0; that is kept. */
static uint32_t cuckoo_alt(const orc_cuckoo *f, uint32_t i, uint32_t tag) {
  if (f->addr.mode == ORC_ADDR_POW2) return (i ^ (tag * ALT_MUL)) & f->addr.block_cnt_mask;
  uint32_t c = f->addr.block_cnt;
  uint32_t s_mod_m = orc_addr_block(&f->addr, tag * ALT_MUL);
  uint32_t x = c - s_mod_m;
  uint32_t mask = (x < i) ? 0xFFFFFFFFu : 0u;
  return (mask & c) + (x - i);
}

/* cuckoofilter_logic.hpp:171-207 */
void orc_cuckoo_index_tag(const orc_cuckoo *f, uint32_t key, uint32_t *i1, uint32_t *i2, uint32_t *tag) {
  *i1 = orc_addr_block(&f->addr, orc_hash(key, 0));
  uint32_t tg = orc_hash(key, 1) & (f->t == 32 ? 0xFFFFFFFFu : ((1u << f->t) - 1u));
  tg += (tg == 0);
  *tag = tg;
  *i2 = cuckoo_alt(f, *i1, tg);
}

typedef struct { uint32_t index, tag; uint8_t used, pad[3]; } victim_rec;

static victim_rec *victim(const orc_cuckoo *f, const void *data) {
  return (victim_rec *)((uint32_t *)data + f->table_words_u32);
}

static uint64_t xs_next(uint64_t *s) {   /* xorshift64* (Vigna 2014) */
  uint64_t x = *s;
  x ^= x >> 12; x ^= x << 25; x ^= x >> 27;
  *s = x;
  return x * 2685821657736338717ull;
}

/* cuckoofilter_table.hpp:185-202 */
static int insert_tag_to_bucket(const orc_cuckoo *f, void *data, uint32_t i, uint32_t tag,
                                int kickout, uint32_t *oldtag, uint64_t *rng) {
  for (uint32_t j = 0; j < f->b; j++) {
    if (orc_cuckoo_read_tag(f, data, i, j) == 0) {
      write_tag(f, data, i, j, tag);
      return 1;
    }
  }
  if (kickout) {
    uint32_t r = (uint32_t)(xs_next(rng) >> 32) % f->b;
    *oldtag = orc_cuckoo_read_tag(f, data, i, r);
    write_tag(f, data, i, r, tag);
  }
  return 0;
}

/* cuckoofilter_logic.hpp:292-337 */
int orc_cuckoo_insert(const orc_cuckoo *f, void *data, const uint32_t *keys,
                      uint64_t n, uint64_t seed) {
  uint64_t rng = seed ? seed : 0x9E3779B97F4A7C15ull;
  int success = 1;
  victim_rec *v = victim(f, data);
  for (uint64_t x = 0; x < n; x++) {
    if (v->used) { success = 0; continue; }
    uint32_t i1, i2, tag;
    orc_cuckoo_index_tag(f, keys[x], &i1, &i2, &tag);
    uint32_t cur = i1, curtag = tag;
    int done = 0;
    for (uint32_t count = 0; count < MAX_KICKS; count++) {
      int kickout = count > 0;
      uint32_t oldtag = 0;
      if (insert_tag_to_bucket(f, data, cur, curtag, kickout, &oldtag, &rng)) { done = 1; break; }
      if (kickout) curtag = oldtag;
      cur = cuckoo_alt(f, cur, curtag);
    }
    if (!done) {
      v->index = cur;
      v->tag = curtag;
      v->used = 1;
    }
  }
  return success;
}

/* cuckoofilter_logic.hpp:346-362 with the exact tag search of
 * cuckoofilter_table_scalar.hpp:48-83 (the SWAR tests are exact). */
int orc_cuckoo_contains(const orc_cuckoo *f, const void *data, uint32_t key) {
  uint32_t i1, i2, tag;
  orc_cuckoo_index_tag(f, key, &i1, &i2, &tag);
  const victim_rec *v = victim(f, data);
  if (v->used && tag == v->tag && (i1 == v->index || i2 == v->index)) return 1;
  for (uint32_t j = 0; j < f->b; j++) {
    if (orc_cuckoo_read_tag(f, data, i1, j) == tag) return 1;
    if (orc_cuckoo_read_tag(f, data, i2, j) == tag) return 1;
  }
  return 0;
}

uint64_t orc_cuckoo_batch_contains(const orc_cuckoo *f, const void *data,
                                   const uint32_t *keys, uint32_t n,
                                   uint32_t *match_pos, uint32_t match_offset) {
  uint64_t cnt = 0;
  for (uint32_t i = 0; i < n; i++)
    if (orc_cuckoo_contains(f, data, keys[i])) match_pos[cnt++] = i + match_offset;
  return cnt;
}

/* cuckoofilter_logic.hpp:496-499, cuckoofilter_table.hpp:255-274 */
uint64_t orc_cuckoo_count_occupied(const orc_cuckoo *f, const void *data) {
  uint64_t cnt = 0;
  for (uint64_t i = 0; i < f->addr.block_cnt; i++)
    for (uint32_t j = 0; j < f->b; j++) cnt += orc_cuckoo_read_tag(f, data, i, j) != 0;
  return cnt + victim(f, data)->used;
}

/* ======================================================================== */
/* Blocked cuckoo filter                                                     */
/* ======================================================================== */

/* blocked_cuckoofilter_multiword_table.hpp:89-110.  Every instantiation the
 * dispatcher offers (blocked_cuckoofilter.hpp:254-297) holds exactly one
 * bucket per word, so a block of block_bytes has block_bytes / word_bytes
 * buckets and bucket i is word i of the block. */
int orc_bcf_init(orc_bcf *f, uint32_t block_bytes, uint32_t t, uint32_t a, uint64_t m) {
  memset(f, 0, sizeof(*f));
  if (!(block_bytes == 8 || block_bytes == 32 || block_bytes == 64 || block_bytes == 128 ||
        block_bytes == 256 || block_bytes == 512)) return ORC_ERR_CONFIG;
  if (!((t == 8 && a == 4) || (t == 8 && a == 8) || (t == 10 && a == 6) || (t == 12 && a == 4) ||
        (t == 16 && a == 2) || (t == 16 && a == 4))) return ORC_ERR_CONFIG;
  f->block_bytes = block_bytes;
  f->t = t; f->a = a; f->m = m;
  f->word_bytes = t * a <= 32 ? 4 : 8;                 /* blocked_cuckoofilter_logic.hpp:280-414 */
  f->bucket_bits = log2_u64(block_bytes / f->word_bytes);
  const uint64_t block_bits = (uint64_t)block_bytes * 8;
  uint32_t mode = is_pow2_u64(m) ? ORC_ADDR_POW2 : ORC_ADDR_MAGIC;  /* blocked_cuckoofilter.hpp:303-312 */
  int rc = orc_addr_init(&f->addr, (m + block_bits - 1) / block_bits, mode);  /* logic.hpp:59-61 */
  if (rc) return rc;
  f->m_actual = (uint64_t)f->addr.block_cnt * block_bits;  /* logic.hpp:262-264 */
  f->word_cnt = f->m_actual / (8ull * f->word_bytes);
  /* word indexes are formed in 32 bits (block_idx << log2(words per block),
   * logic.hpp:76,106): larger filters would wrap */
  if (f->word_cnt > (1ull << 32)) return ORC_ERR_SIZE;
  f->size_u32 = (f->m_actual + 31) / 32;                  /* blocked_cuckoofilter.hpp:435-438 */
  const uint32_t req = mode == ORC_ADDR_MAGIC ? 32u : f->addr.block_cnt_log2;  /* block_addressing_logic.hpp:131,230 */
  f->hash_shift = req + t + f->bucket_bits <= 32 ? req : 32u;
  return ORC_OK;
}

static uint64_t bcf_bucket_mask(const orc_bcf *f) {     /* multiword_table.hpp:100,111 */
  const uint32_t bits = f->t * f->a;
  return bits == f->word_bytes * 8 ? ~0ull >> (64 - bits) : (1ull << bits) - 1;
}

static uint64_t bcf_read(const orc_bcf *f, const void *block, uint32_t i) {   /* :116-123 */
  return f->word_bytes == 4 ? ((const uint32_t *)block)[i] : ((const uint64_t *)block)[i];
}
static void bcf_write(const orc_bcf *f, void *block, uint32_t i, uint64_t v) { /* :127-136 */
  if (f->word_bytes == 4) ((uint32_t *)block)[i] = (uint32_t)v;
  else ((uint64_t *)block)[i] = v;
}
static uint32_t bcf_tag_at(const orc_bcf *f, uint64_t bucket, uint32_t j) {  /* :146-150 */
  return (uint32_t)((bucket >> (f->t * j)) & ((1u << f->t) - 1));
}

/* packed_value<word, t>::contains (blocked_cuckoofilter_util.hpp:14-88): the
 * SWAR "has a field equal to n" test, with the reference's own field sets.
 * With 32-bit words and 16-bit tags the reference's constants are 64-bit, so
 * that test runs in 64 bits on the zero-extended word. */
static int bcf_has(const orc_bcf *f, uint64_t x, uint32_t n) {
  uint32_t fields;
  switch (f->t) {
    case 8: fields = f->word_bytes * 8 / 8; break;  /* 4 or 8 */
    case 10: fields = 6; break;
    case 12: fields = 5; break;
    default: fields = 4; break;                      /* 16 */
  }
  uint64_t L = 0;
  for (uint32_t i = 0; i < fields; i++) L |= 1ull << (f->t * i);
  const uint64_t H = L << (f->t - 1);
  if (f->t == 8 && f->word_bytes == 4) {
    const uint32_t y = (uint32_t)x ^ (n * (uint32_t)L);
    return ((y - (uint32_t)L) & ~y & (uint32_t)H) != 0;
  }
  const uint64_t y = x ^ ((uint64_t)n * L);
  return ((y - L) & ~y & H) != 0;
}

/* Block index, the hash the block's cuckoo table works on, and the block's
 * base address (blocked_cuckoofilter_logic.hpp:73-82,103-111). */
static uint32_t bcf_block_hash(const orc_bcf *f, uint32_t key, uint32_t *hv) {
  const uint32_t h = key * kMul[1];                      /* knuth_32_alt: hash.hpp:73-83 */
  const uint32_t blk = orc_addr_block(&f->addr, h);
  *hv = f->hash_shift < 32 ? h << f->hash_shift : key * kMul[0];  /* knuth_32: hash.hpp:59-69 */
  return blk;
}

/* blocked_cuckoofilter_block_logic.hpp:45-72,128-133 */
static uint32_t bcf_bucket(const orc_bcf *f, uint32_t hv) {
  return f->bucket_bits ? hv >> (32 - f->bucket_bits) : 0u;
}
static uint32_t bcf_tag(const orc_bcf *f, uint32_t hv) {
  uint32_t tag = (hv >> (32 - f->bucket_bits - f->t)) & ((1u << f->t) - 1);
  return tag + (tag == 0);
}
static uint32_t bcf_alt(const orc_bcf *f, uint32_t i, uint32_t tag) {
  return f->bucket_bits ? i ^ ((tag * ALT_MUL) >> (32 - f->bucket_bits)) : i;
}

void orc_bcf_locate(const orc_bcf *f, uint32_t key, uint32_t *block, uint32_t *b1, uint32_t *b2,
                    uint32_t *tag) {
  uint32_t hv;
  *block = bcf_block_hash(f, key, &hv);
  *b1 = bcf_bucket(f, hv);
  *tag = bcf_tag(f, hv);
  *b2 = bcf_alt(f, *b1, *tag);
}

#define BCF_OVERFLOW_TAG 0xFFFFFFFFu   /* multiword_table.hpp:110 */
#define BCF_RELOCATIONS 10u            /* block_logic.hpp:108 */

/* insert_tag (multiword_table.hpp:203-224) and, with relocate, its kicking
 * twin insert_tag_relocate (:176-200): the first slot holding the tag or empty
 * takes it; a full bucket hands back its own tag (insert_tag) or swaps it with
 * a random slot and hands back the tag it displaced. */
static uint32_t bcf_insert_tag(const orc_bcf *f, void *block, uint32_t i, uint32_t tag, int relocate,
                               uint64_t *rng) {
  uint64_t bucket = bcf_read(f, block, i);
  if (bucket == bcf_bucket_mask(f)) return BCF_OVERFLOW_TAG;
  for (uint32_t j = 0; j < f->a; j++) {
    const uint32_t x = bcf_tag_at(f, bucket, j);
    if (x == tag) return 0;
    if (x == 0) {
      bcf_write(f, block, i, bucket | ((uint64_t)tag << (f->t * j)));
      return 0;
    }
  }
  if (!relocate) return tag;
  const uint32_t r = (uint32_t)(xs_next(rng) >> 32) % f->a;
  const uint32_t old = bcf_tag_at(f, bucket, r);
  bcf_write(f, block, i, bucket ^ ((uint64_t)(old ^ tag) << (f->t * r)));
  return old;
}

/* blocked_cuckoofilter_block_logic.hpp:96-118 */
static void bcf_block_insert(const orc_bcf *f, void *block, uint32_t i, uint32_t tag, uint64_t *rng) {
  uint32_t old = bcf_insert_tag(f, block, i, tag, 0, rng);
  if (old == 0 || old == BCF_OVERFLOW_TAG) return;
  uint32_t cur = bcf_alt(f, i, tag), curtag = tag;
  for (uint32_t c = 0; c < BCF_RELOCATIONS; c++) {
    old = bcf_insert_tag(f, block, cur, curtag, 1, rng);
    if (old == 0 || old == BCF_OVERFLOW_TAG) return;
    curtag = old;
    cur = bcf_alt(f, cur, curtag);
  }
  bcf_write(f, block, cur, bcf_bucket_mask(f));   /* mark_overflow: multiword_table.hpp:140-142 */
}

static void *bcf_block_ptr(const orc_bcf *f, const void *data, uint32_t blk) {
  return (uint8_t *)data + (uint64_t)blk * f->block_bytes;
}

void orc_bcf_insert(const orc_bcf *f, void *data, const uint32_t *keys, uint64_t n, uint64_t seed) {
  uint64_t rng = seed ? seed : 0x9E3779B97F4A7C15ull;
  for (uint64_t x = 0; x < n; x++) {
    uint32_t hv;
    const uint32_t blk = bcf_block_hash(f, keys[x], &hv);
    bcf_block_insert(f, bcf_block_ptr(f, data, blk), bcf_bucket(f, hv), bcf_tag(f, hv), &rng);
  }
}

/* contains_hash (block_logic.hpp:151-158) with find_tag<table, 1>
 * (multiword_table.hpp:51-67): an overflowed bucket answers every key. */
int orc_bcf_contains(const orc_bcf *f, const void *data, uint32_t key) {
  uint32_t blk, i1, i2, tag;
  orc_bcf_locate(f, key, &blk, &i1, &i2, &tag);
  const void *block = bcf_block_ptr(f, data, blk);
  const uint64_t b1 = bcf_read(f, block, i1), b2 = bcf_read(f, block, i2);
  const uint64_t ovf = bcf_bucket_mask(f);
  return b1 == ovf || b2 == ovf || bcf_has(f, b1, tag) || bcf_has(f, b2, tag);
}

/* blocked_cuckoofilter_logic.hpp:120-170 (scalar batch path) */
uint64_t orc_bcf_batch_contains(const orc_bcf *f, const void *data, const uint32_t *keys,
                                uint32_t n, uint32_t *match_pos, uint32_t match_offset) {
  uint64_t cnt = 0;
  for (uint32_t i = 0; i < n; i++)
    if (orc_bcf_contains(f, data, keys[i])) match_pos[cnt++] = i + match_offset;
  return cnt;
}

/* ======================================================================== */
/* Classic Bloom filter                                                      */
/* ======================================================================== */

/* bloomfilter_logic.hpp:62-64: one addressing "block" per 32-bit word.  The
 * bit index is (h >> (32 - 5 - addressing bits)) & 31 (:105,138), a shift the
 * C++ leaves undefined once the addressing bits exceed 27.  Restated as the
 * reference compiles (g++ 13, x86-64, -O2; pinned by tests against
 * oracle/_ref): with POW2 the shift count is a run-time value and x86 takes it
 * mod 32; with MAGIC the addressing bits are the constant 32 and the compiler
 * folds the bit index to 0. */
int orc_cbf_init(orc_cbf *f, uint32_t k, uint64_t m, uint32_t mode) {
  memset(f, 0, sizeof(*f));
  if (k > 17) return ORC_ERR_CONFIG;   /* dyn::mul32 throws for hash_no > 16 (hash_family.hpp:295-297) */
  f->k = k;
  f->m = m;
  int rc = orc_addr_init(&f->addr, (m + 31) / 32, mode);
  if (rc) return rc;
  f->word_cnt = f->addr.block_cnt;                      /* :84-87 */
  f->m_actual = (uint64_t)f->addr.block_cnt * 32;       /* :74-77 */
  if (mode == ORC_ADDR_MAGIC) {
    f->bit_shift = 0;
    f->bit_mask = 0;
  } else {
    f->bit_shift = (27u - f->addr.block_cnt_log2) & 31u;
    f->bit_mask = 31;
  }
  return ORC_OK;
}

static uint32_t cbf_bit(const orc_cbf *f, uint32_t h) { return (h >> f->bit_shift) & f->bit_mask; }

/* :94-121 */
void orc_cbf_insert(const orc_cbf *f, void *data, const uint32_t *keys, uint64_t n) {
  uint32_t *w = (uint32_t *)data;
  for (uint64_t x = 0; x < n; x++) {
    for (uint32_t i = 0; i < f->k; i++) {
      const uint32_t h = keys[x] * kMul[i];            /* dyn::mul32 (hash_family.hpp:271-299) */
      w[orc_addr_block(&f->addr, h)] |= 1u << cbf_bit(f, h);
    }
  }
}

/* :127-144, with its early out */
int orc_cbf_contains(const orc_cbf *f, const void *data, uint32_t key) {
  const uint32_t *w = (const uint32_t *)data;
  for (uint32_t i = 0; i < f->k; i++) {
    const uint32_t h = key * kMul[i];
    if (!((w[orc_addr_block(&f->addr, h)] >> cbf_bit(f, h)) & 1u)) return 0;
  }
  return 1;
}

/* :188-208 */
uint64_t orc_cbf_batch_contains(const orc_cbf *f, const void *data, const uint32_t *keys,
                                uint32_t n, uint32_t *match_pos, uint32_t match_offset) {
  uint64_t cnt = 0;
  for (uint32_t i = 0; i < n; i++)
    if (orc_cbf_contains(f, data, keys[i])) match_pos[cnt++] = i + match_offset;
  return cnt;
}
