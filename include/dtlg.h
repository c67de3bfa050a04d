/*
 * dtlg.h -- C ABI of the B200-native DTL filter build/probe library (libdtlg.so).
 *
 * Drop-in boundary for the filter path of peterboncz/bloomfilter-bsd ("dtl").
 * The reference exposes that path as the C++ interface dtl::filter::filter_base
 * (src/dtl/filter/filter_base.hpp:11-62), implemented by bbf_32, bbf_64,
 * zbbf_32, zbbf_64 and cf, constructed by config through the dtl::filter::filter
 * facade (src/dtl/filter/filter.hpp:42-72,166-169).  Every entry point below
 * names the reference member it replaces.
 *
 * Conventions
 *  - Plain pointers and sizes only; no C++ or torch types cross this boundary.
 *  - Unless a name ends in _host, every data pointer is a DEVICE pointer on the
 *    current CUDA device, and work is enqueued on `stream` (0 = legacy default).
 *  - As in the reference, the caller owns the filter words (filter.hpp:92-119):
 *    allocate dtlg_alloc_words_u64() 64-bit words, zero them, pass them in.
 *  - Errors are returned as dtlg_status; nothing is thrown across the ABI.
 *  - Results are bit-identical to the reference's scalar contains path:
 *    the same filter words after batch_insert (Bloom) and the same ascending
 *    match positions i + match_offset (32-bit wrap) from batch_contains.
 */
#ifndef DTLG_H
#define DTLG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* dtlg_stream_t; /* == cudaStream_t */

typedef enum dtlg_status {
  DTLG_OK = 0,
  DTLG_ERR_INVALID_CONFIG = 1, /* reference: std::invalid_argument / runtime_error from the ctor */
  DTLG_ERR_SIZE = 2,           /* reference: std::logic_error "block count must not exceed 2^32" */
  DTLG_ERR_NULL = 3,           /* a required pointer is NULL */
  DTLG_ERR_ALIGNMENT = 4,      /* filter words not 16-byte aligned */
  DTLG_ERR_CUDA = 5,           /* a CUDA call failed; see dtlg_last_cuda_error() */
  DTLG_ERR_ALLOC = 6,          /* device or pinned allocation failed */
  DTLG_ERR_CUCKOO_FULL = 7,    /* reference: cuckoo batch_insert returned false */
  DTLG_ERR_TIMEOUT = 8,        /* a bounded device wait gave up (look-back / queue) */
  DTLG_ERR_WORKSPACE = 9,      /* caller workspace too small */
  DTLG_ERR_UNSUPPORTED = 10    /* operation not defined for this filter kind */
} dtlg_status;

/* Mirrors dtl::blocked_bloomfilter_config
 * (src/dtl/filter/blocked_bloomfilter/blocked_bloomfilter_config.hpp:11-18).
 * addr_mode is informational, as in the reference: the addressing is POW2 iff
 * m is a power of two (blocked_bloomfilter.hpp:234-242). */
typedef struct dtlg_bloom_config {
  uint32_t k;                  /* bits set per key, 1..16 (default 8) */
  uint32_t word_size;          /* bytes per word, 4 or 8 (default 4) */
  uint32_t word_cnt_per_block; /* 1,2,4,8,16 (default 1) */
  uint32_t sector_cnt;         /* 1,2,4,8,16 (default 1) */
  uint32_t addr_mode;          /* 0 = POW2, 1 = MAGIC (ignored on create) */
  uint32_t zone_cnt;           /* 1 = not zoned; 2,4,8 = zoned (default 1) */
} dtlg_bloom_config;

/* Mirrors dtl::cuckoofilter::config
 * (src/dtl/filter/cuckoofilter/cuckoofilter_config.hpp:13-16). */
typedef struct dtlg_cuckoo_config {
  uint32_t bits_per_tag;    /* 4, 8, 12, 16, 32 */
  uint32_t tags_per_bucket; /* 1, 2, 4 */
  uint32_t addr_mode;       /* informational, as above */
} dtlg_cuckoo_config;

/* Mirrors the constructor arguments of dtl::bcf, the blocked cuckoo filter
 * (src/dtl/filter/bcf.hpp:56: block_size_bytes = 64, tag_size_bits = 16,
 * associativity = 4).  block_size_bytes: 8, 32, 64, 128, 256, 512; (tag bits,
 * associativity): (8,4) (8,8) (10,6) (12,4) (16,2) (16,4)
 * (blocked_cuckoofilter.hpp:254-297).  Addressing is POW2 iff m is a power of
 * two (:303-312). */
typedef struct dtlg_blocked_cuckoo_config {
  uint32_t block_size_bytes;
  uint32_t tag_size_bits;
  uint32_t associativity;
} dtlg_blocked_cuckoo_config;

/* Mirrors dtl::bloomfilter_logic<uint32_t, addr_mode>(m, k), the classic
 * Bloom filter (src/dtl/filter/bloomfilter/bloomfilter_logic.hpp:22-64): one
 * bit in each of k 32-bit words.  The addressing is the template argument
 * there (no dispatcher), so it is explicit here: 0 = POW2, 1 = MAGIC. */
typedef struct dtlg_classic_bloom_config {
  uint32_t k;         /* 0..17 (hash functions C[0..k-1], hash_family.hpp:271-299) */
  uint32_t addr_mode;
} dtlg_classic_bloom_config;

typedef struct dtlg_filter dtlg_filter;

/* ---- construction (filter.hpp:42-72; bbf_32.hpp:53, zbbf_*.hpp, cf.hpp) ---- */
dtlg_status dtlg_bloom_create(const dtlg_bloom_config* cfg, uint64_t m_bits, dtlg_filter** out);
dtlg_status dtlg_cuckoo_create(const dtlg_cuckoo_config* cfg, uint64_t m_bits, dtlg_filter** out);
/* dtl::bcf::bcf(m, block_size_bytes, tag_size_bits, associativity)
 * (bcf.hpp:56, bcf.cpp:24-25).  dtl::bcf is not a filter_base (bcf.hpp:11):
 * its size() counts 32-bit words; dtlg_size() here counts 64-bit words (half
 * of that; blocks are >= 8 bytes) like every other kind. */
dtlg_status dtlg_blocked_cuckoo_create(const dtlg_blocked_cuckoo_config* cfg, uint64_t m_bits,
                                       dtlg_filter** out);
/* dtl::bloomfilter_logic<uint32_t, A>::bloomfilter_logic(m, k)
 * (bloomfilter_logic.hpp:62-64).  k > 17 is rejected here; the reference
 * throws from inside its noexcept insert / contains (std::terminate). */
dtlg_status dtlg_classic_bloom_create(const dtlg_classic_bloom_config* cfg, uint64_t m_bits, dtlg_filter** out);
void dtlg_destroy(dtlg_filter* f);

/* ---- sizes and name ---- */
/* filter_base::size_in_bytes() (filter_base.hpp:52) */
uint64_t dtlg_size_in_bytes(const dtlg_filter* f);
/* filter_base::size(): filter size in 64-bit words (filter_base.hpp:56) */
uint64_t dtlg_size(const dtlg_filter* f);
/* 64-bit words the caller must allocate (zeroed): size(), plus for cuckoo the
 * victim-cache record the reference keeps past size() (cuckoofilter_logic.hpp:
 * 145-157) and read slack. */
uint64_t dtlg_alloc_words_u64(const dtlg_filter* f);
/* filter_base::name(): the reference's JSON description (filter_base.hpp:48,
 * blocked_bloomfilter.hpp:372-390, zoned_blocked_bloomfilter.hpp:358-378,
 * cuckoofilter.hpp:335-343, blocked_cuckoofilter.hpp:445-454).  Writes a NUL-terminated string; returns its
 * length (excluding NUL) or the required length if cap is too small. */
size_t dtlg_name(const dtlg_filter* f, char* buf, size_t cap);
/* Introspection: 0 = Bloom, 1 = zoned Bloom, 2 = cuckoo, 3 = blocked cuckoo,
 * 4 = classic Bloom;
 * block (bucket) count; 1 if MAGIC addressing. */
int dtlg_kind(const dtlg_filter* f);
uint64_t dtlg_block_cnt(const dtlg_filter* f);
int dtlg_is_magic(const dtlg_filter* f);

/* ---- build: filter_base::batch_insert (filter_base.hpp:26) ---- */
/* Bloom, classic Bloom and blocked cuckoo: always DTLG_OK on valid input
 * (bbf_32.cpp:41-45, bloomfilter_logic.hpp:115-121,
 * bcf.cpp:36-40; a blocked cuckoo key that finds no slot marks its bucket
 * overflowed, block_logic.hpp:117).  Cuckoo: returns
 * DTLG_ERR_CUCKOO_FULL when some key could not be placed (the reference's
 * `false`, cuckoofilter_logic.hpp:330-337); *failed_out (optional) gets the
 * number of keys lost.  Synchronous w.r.t. `stream` for cuckoo only. */
dtlg_status dtlg_batch_insert(const dtlg_filter* f, uint64_t* filter_words, const uint32_t* keys,
                              uint32_t key_cnt, uint64_t* failed_out, dtlg_stream_t stream);

/* ---- probe: filter_base::batch_contains (filter_base.hpp:42-45) ---- */
/* Writes the positions i + match_offset of matching keys, ascending, to
 * match_positions (capacity >= key_cnt) and the match count to *match_cnt
 * (HOST pointer); blocks until the count is known. */
dtlg_status dtlg_batch_contains(const dtlg_filter* f, const uint64_t* filter_words,
                                const uint32_t* keys, uint32_t key_cnt, uint32_t* match_positions,
                                uint32_t match_offset, uint64_t* match_cnt, dtlg_stream_t stream);
/* Fully asynchronous form: the count goes to *match_cnt_dev (DEVICE pointer).
 * The asynchronous forms (_async, _ws, _gather, _noalloc) cannot return
 * DTLG_ERR_TIMEOUT, since the status is known only on the device: when one of
 * the probe's bounded device waits gives up, *match_cnt_dev is set to
 * UINT64_MAX and the positions are invalid.  Read the count as
 * DTLG_ERR_TIMEOUT in that case (dtlg_batch_contains does so itself). */
dtlg_status dtlg_batch_contains_async(const dtlg_filter* f, const uint64_t* filter_words,
                                      const uint32_t* keys, uint32_t key_cnt,
                                      uint32_t* match_positions, uint32_t match_offset,
                                      uint64_t* match_cnt_dev, dtlg_stream_t stream);
/* Same, with a caller-provided device workspace of at least
 * dtlg_probe_workspace_size(key_cnt) bytes (no allocation inside). */
size_t dtlg_probe_workspace_size(uint32_t key_cnt);
dtlg_status dtlg_batch_contains_ws(const dtlg_filter* f, const uint64_t* filter_words,
                                   const uint32_t* keys, uint32_t key_cnt, uint32_t* match_positions,
                                   uint32_t match_offset, uint64_t* match_cnt_dev, void* workspace,
                                   size_t workspace_bytes, dtlg_stream_t stream);

/* Probe -> gather, the step after the reference's batch_contains in a
 * semi-join (the per-tuple work tw of model/cost_fn.hpp:159-166): as
 * dtlg_batch_contains_ws, and for the match of key i at list slot j also
 * out_cols[c][j] = cols[c][i] for each of n_cols (<= 4) payload columns of
 * col_bytes[c] = 4 or 8 bytes (device arrays of n rows / capacity >= n rows).
 * match_positions may be NULL when n_cols > 0.  Counterpart: none fused; the
 * reference's callers gather from the position list afterwards. */
dtlg_status dtlg_batch_contains_gather(const dtlg_filter* f, const uint64_t* filter_words, const uint32_t* keys,
                                       uint32_t key_cnt, uint32_t n_cols, const void* const* cols,
                                       const uint32_t* col_bytes, void* const* out_cols, uint32_t* match_positions,
                                       uint32_t match_offset, uint64_t* match_cnt_dev, void* workspace,
                                       size_t workspace_bytes, dtlg_stream_t stream);
/* Probe tuning of one filter (set by the autotuner, dtlg_autotune_probe):
 * mode 0 = automatic, 1 = one fused kernel (probe + ordered compaction),
 * 2 = two streaming kernels (match bitmask, then compaction), 3 = partitioned
 * (keys sorted into ~8 MiB block ranges; Bloom and blocked cuckoo filters),
 * 4 = match bitmask against a copy of the filter in every CTA's shared memory
 * (Bloom and classic Bloom filters of at most 192 KiB); a plan the filter does
 * not offer falls back to 2.  Automatic: 1 below 2^20 keys; 3 for filters
 * beyond 160 MiB, except Bloom layouts measured faster in plan 2 (words picked
 * by the hash, s < w, up to 256 MiB; blocks under 32 bytes up to 240 MiB;
 * zoned u32 up to 224 MiB); else 2.  variant selects the register budget of
 * the bitmask and pair kernels (-1 = automatic: 0 for the pair probe of Bloom
 * filters and for plan 2 in the exceptions above, else 1; 0 = 32 registers at
 * 8 CTAs/SM, 1 = 64 registers at 4 CTAs/SM).  Results never change.
 * (The reference's counterpart is its per-config SIMD unroll factor,
 * blocked_bloomfilter_tune.hpp:21-56.) */
dtlg_status dtlg_set_probe_options(dtlg_filter* f, int mode, int variant);
/* Build plan of a blocked Bloom or blocked cuckoo filter (no counterpart in
 * the reference, whose batch_insert is one loop): 0 = automatic (2 for Bloom
 * filters beyond 80 MiB and batches of >= 2^20 keys, else 1), 1 = one kernel of
 * global atomics, 2 = keys first grouped by ~8 MiB block range (the
 * partitioned probe's partition, ~8.3 bytes per key of workspace from the
 * library's stream-ordered pool; without room there, plan 1), then inserted
 * range by range so the atomics hit L2.  Bloom filter
 * words are the same under every plan; blocked cuckoo builds are randomised
 * under both (as the reference's); other filter kinds ignore it. */
dtlg_status dtlg_set_build_options(dtlg_filter* f, int mode);
/* Block-range passes of the two-kernel probe (0 = automatic, 1..16).  Random
 * probes over more than ~256 MiB of filter exceed the GPU's address-translation
 * reach; probing one block range per pass keeps each pass within it. */
dtlg_status dtlg_set_probe_passes(dtlg_filter* f, int passes);
/* Number of kernels one batch_contains of key_cnt keys launches with the
 * current options (fused: 1; two-kernel: block-range passes + compaction). */
int dtlg_probe_kernel_count(const dtlg_filter* f, uint32_t key_cnt);

/* Sets the L2 fetch granularity hint of the CURRENT device's context
 * (cudaLimitMaxL2FetchGranularity; 0, 32, 64 or 128 bytes) and returns the
 * value in effect in *in_effect.  Random 32/64-byte filter reads waste HBM
 * bandwidth when every miss fills a 128-byte line.  The limit belongs to this
 * process's context only and ends with it. */
dtlg_status dtlg_set_l2_fetch_granularity(int bytes, int* in_effect);

/* Probe autotuner, the counterpart of the reference's calibrate() tuners
 * (blocked_bloomfilter_tune_impl.hpp:162-268, cuckoofilter_tune_impl.hpp:
 * 118-225), which time SIMD unroll factors: times every probe plan (fused;
 * bitmask kernel x register budget x block-range passes; partitioned beyond
 * 32 MiB; shared-memory up to 192 KiB) on these keys, `reps` runs each, keeps the
 * fastest on the handle (as dtlg_set_probe_options / _passes would) and
 * reports it.  All plans must agree on the match count (else DTLG_ERR_CUDA).
 * match_positions: device, capacity >= n (scratch). */
typedef struct dtlg_probe_plan {
  int mode;                      /* 1 fused, 2 bitmask + compaction, 3 partitioned, 4 shared memory */
  int variant;                   /* bitmask kernel register budget (-1: n/a) */
  int passes;                    /* block-range passes of mode 2 (0: automatic) */
  float ms;                      /* median time of one probe of the n keys */
  float gkeys_per_s;
} dtlg_probe_plan;
dtlg_status dtlg_autotune_probe(dtlg_filter* f, const uint64_t* filter_words, const uint32_t* keys, uint32_t n,
                                uint32_t* match_positions, int reps, dtlg_stream_t stream, dtlg_probe_plan* best);

/* ---- probe without any allocation (no counterpart in the reference) ----
 * For callers that cannot call cudaMalloc -- a query engine whose device
 * memory is all owned by its own buffer manager, a plugin inside a host
 * application that has claimed the GPU's memory, a latency-critical path that
 * cannot afford an allocation's synchronization.  Same result as
 * dtlg_batch_contains_async; the count goes to *match_cnt_dev (DEVICE).  The
 * probe's scratch (tile queue + look-back words) lives in one static device
 * array of about 128 KiB per GPU, held until exit; key_cnt above
 * DTLG_NOALLOC_MAX_KEYS is rejected with DTLG_ERR_WORKSPACE.  The first call
 * on each device looks the array's address up (make that first call before
 * any stream capture); the address is kept for the life of the process, so
 * the entry point must not be used after a cudaDeviceReset of that device.
 * All calls share the array: calls that overlap on the GPU race and must be
 * serialized by the caller.  It always runs the single fused probe kernel
 * (its scratch has no room for a match bitmask or key pairs) and ignores the
 * plan of dtlg_set_probe_options / dtlg_autotune_probe: the results are the
 * same, but filters far beyond L2 probe about 2-2.5x slower than with the
 * bitmask or partitioned plans that dtlg_batch_contains_async picks there.
 * A bounded device wait that gives up leaves UINT64_MAX in *match_cnt_dev. */
#define DTLG_NOALLOC_MAX_KEYS (1u << 26)
dtlg_status dtlg_batch_contains_noalloc(const dtlg_filter* f, const uint64_t* filter_words,
                                        const uint32_t* keys, uint32_t key_cnt,
                                        uint32_t* match_positions, uint32_t match_offset,
                                        uint64_t* match_cnt_dev, dtlg_stream_t stream);

/* ---- many filters at once (no counterpart in the reference) ----
 * A query with one filter per partition or semi-join calls batch_insert and
 * batch_contains once per filter in the reference (filter_base.hpp:26,42-45).
 * dtlg_batch_prepare turns such a list of calls into device tables (it
 * allocates and copies; the buffers named by the items must stay valid and
 * unchanged); dtlg_batch_run then builds and probes all filters in ONE
 * persistent kernel (optionally replayed as a CUDA graph).  Results are those
 * of the per-filter calls: each item's filter words after inserting its build
 * keys, and its probe keys' ascending match positions + count (DEVICE).
 * Bloom filters of the compiled menu (u64 w=8 s=8 k=8; zoned u64 w=8 and u32
 * w=16 with z=2/4, k=8; u32 w=1 k=4/8) run inside the persistent kernel;
 * other Bloom configs (or keys not 16-byte aligned) run as separate launches
 * in the same stream / graph.  Cuckoo filters: DTLG_ERR_UNSUPPORTED. */
typedef struct dtlg_batch_item {
  const dtlg_filter* filter;
  uint64_t* filter_words;        /* device, as for dtlg_batch_insert */
  const uint32_t* build_keys;    /* device */
  uint32_t n_build;
  const uint32_t* probe_keys;    /* device */
  uint32_t n_probe;
  uint32_t* match_positions;     /* device, capacity >= n_probe */
  uint32_t match_offset;
  uint64_t* match_cnt;           /* device */
} dtlg_batch_item;
typedef struct dtlg_batch dtlg_batch;
dtlg_status dtlg_batch_prepare(const dtlg_batch_item* items, uint32_t n_items, int use_graph, dtlg_batch** out);
dtlg_status dtlg_batch_run(dtlg_batch* b, dtlg_stream_t stream);
/* CTAs per SM of the persistent kernel (0 = as many as fit); set by the autotuner. */
dtlg_status dtlg_batch_set_ctas_per_sm(dtlg_batch* b, int ctas_per_sm);
/* Build staging: 0 = every filter of at most 2048 ranges of 32 KiB is built
 * range by range in shared memory from key buckets (default), 1 = all filters
 * insert with global atomics.  Results are identical; set by the autotuner. */
dtlg_status dtlg_batch_set_staging(dtlg_batch* b, int staging);
uint32_t dtlg_batch_staged_count(const dtlg_batch* b);
/* Autotuner: times every (staging, CTAs per SM) choice over `reps` runs of
 * the batch (runs are idempotent: OR-builds and the same match lists) and
 * keeps the fastest. */
typedef struct dtlg_batch_plan {
  int staging;
  int ctas_per_sm;
  float ms;                      /* median time of one run */
} dtlg_batch_plan;
dtlg_status dtlg_batch_autotune(dtlg_batch* b, int reps, dtlg_stream_t stream, dtlg_batch_plan* best);
int dtlg_batch_kernel_count(const dtlg_batch* b);
uint32_t dtlg_batch_fallback_count(const dtlg_batch* b);
void dtlg_batch_destroy(dtlg_batch* b);

/* ---- configuration choice: exhaustive calibrated search and MLP cost model ----
 * Replaces the reference's model/ directory: cost_fn::overhead
 * (model/cost_fn.hpp:150-160) minimised over m by model::optimizer
 * (model/optimizer.hpp:25-140) for every configuration, as
 * build_skyline_matrix does (tool/calibration/src/skyline_matrix_builder.cpp:
 * 88-115).  Host memory throughout; the lookup times come from GPU calibration
 * runs (t per key at log2-spaced filter sizes).
 *   cost(c, bpk) = t_c(n * bpk / 8 bytes) + ns_per_match * (h + (1 - h) f)
 *                  + work_ns * (1 - h) f,    f = fpr_c(bpk) <= fpr_target */
typedef struct dtlg_cost_tables {
  uint32_t n_cand;              /* C candidate configurations */
  uint32_t n_bpk;               /* K bits-per-key grid points */
  const double* bits_per_key;   /* [K], ascending */
  const double* fpr;            /* [C*K]; +inf where the layout cannot hold the keys */
  uint32_t n_size;              /* S calibrated filter sizes */
  double log2_bytes_first;      /* size i is 2^(first + i * step) bytes */
  double log2_bytes_step;
  const double* ns_per_key;     /* [C*S] probe time per key */
  double ns_per_match;          /* added time per matching key */
  double l2_budget_bytes;       /* size limit of l2_resident queries */
  /* [C*S] added time per key that loads the second half of its block (the
   * probe tests the first half first and skips the rest when it fails);
   * NULL: no second part.  A key loads it when it is a member (h) or a
   * non-member that passes the first half, q = sqrt(f) (the half's false-
   * positive rate where both halves are alike; an upper bound otherwise):
   *   t_c = ns_per_key + (h + (1 - h) q) ns_second */
  const double* ns_second;
} dtlg_cost_tables;
typedef struct dtlg_cost_query {
  double log2_n;                /* build keys */
  double fpr_target;            /* the filter's FPR must not exceed it */
  double hit_ratio;             /* share of probe keys in the build set */
  double work_ns;               /* downstream work per tuple that passes the filter */
  uint32_t l2_resident;         /* 1: the filter must fit l2_budget_bytes */
} dtlg_cost_query;
/* Every candidate's least cost over the grid (cand_cost / cand_bpk [Q*C], may
 * be NULL; +inf / NaN when infeasible) and the best candidate (best = -1 when
 * none is feasible).  threads <= 0: all host cores. */
dtlg_status dtlg_cost_search(const dtlg_cost_tables* t, const dtlg_cost_query* queries, uint32_t n_queries,
                             double* cand_cost, double* cand_bpk, int32_t* best, double* best_cost,
                             double* best_bpk, int threads);
/* The cost of given choices (candidate, bits-per-key grid index); +inf if infeasible. */
dtlg_status dtlg_cost_eval(const dtlg_cost_tables* t, const dtlg_cost_query* queries, uint32_t n_queries,
                           const int32_t* cand, const uint32_t* bpk_index, double* cost);

/* The MLP cost model: `hidden_layers` ReLU layers of `width` FP32 units and a
 * linear output layer, trained and evaluated by this library's own kernels on
 * the current device (forward, backward, Adam).  Parameters: for each layer
 * W [in x out] row-major then b [out], back to back.  Device pointers for
 * x / t / w / y / batch_rows / loss; host pointers for get/set_params.
 * Loss = (1/N) sum w_ij (y_ij - t_ij)^2.  No counterpart in the reference. */
typedef struct dtlg_mlp dtlg_mlp;
dtlg_status dtlg_mlp_create(uint32_t n_in, uint32_t width, uint32_t hidden_layers, uint32_t n_out,
                            uint32_t max_batch, dtlg_mlp** out);
void dtlg_mlp_destroy(dtlg_mlp* m);
uint64_t dtlg_mlp_param_count(const dtlg_mlp* m);
dtlg_status dtlg_mlp_set_params(dtlg_mlp* m, const float* params_host);  /* also resets Adam state */
dtlg_status dtlg_mlp_get_params(const dtlg_mlp* m, float* params_host);
dtlg_status dtlg_mlp_get_grads(const dtlg_mlp* m, float* grads_host);
dtlg_status dtlg_mlp_forward(dtlg_mlp* m, const float* x, uint32_t n, float* y, dtlg_stream_t stream);
/* Loss and gradients of one batch of n <= max_batch rows; *loss (device) = L. */
dtlg_status dtlg_mlp_loss_grad(dtlg_mlp* m, const float* x, const float* t, const float* w, uint32_t n,
                               float* loss, dtlg_stream_t stream);
dtlg_status dtlg_mlp_adam_step(dtlg_mlp* m, float lr, float beta1, float beta2, float eps, dtlg_stream_t stream);
/* `steps` Adam steps (beta 0.9 / 0.999, eps 1e-8, cosine learning-rate decay
 * lr_start -> lr_end) on batches of `batch` rows: step s uses rows
 * batch_rows[s*batch .. s*batch+batch-1] of (x, t, w); loss_curve[s] = its loss. */
dtlg_status dtlg_mlp_train(dtlg_mlp* m, const float* x, const float* t, const float* w, uint32_t n_rows,
                           const uint32_t* batch_rows, uint32_t batch, uint32_t steps, float lr_start,
                           float lr_end, float* loss_curve, dtlg_stream_t stream);
/* Forward (into y_scratch [n x n_out]) and per row the argmin of the first
 * n_cand outputs (choice) and output n_cand + choice (aux, may be NULL). */
dtlg_status dtlg_mlp_choose(dtlg_mlp* m, const float* x, uint32_t n, uint32_t n_cand, float* y_scratch,
                            int32_t* choice, float* aux, dtlg_stream_t stream);

/* ---- sharded builds (several GPUs) ----
 * dst[i] |= src[j * src_stride + i] for i < n_words, j < n_src (device
 * pointers): the OR that combines partial Bloom filters built from shards of
 * the keys.  Counterpart: the reference replicates a finished filter per NUMA
 * node (filter.hpp:128-152) and has no sharded build. */
dtlg_status dtlg_or_words(uint64_t* dst, const uint64_t* src, uint64_t n_words, uint32_t n_src, uint64_t src_stride,
                          dtlg_stream_t stream);

/* ---- per-device replicas (filter.hpp:98-152) ----
 * Copies n_words filter words from src on src_device to dst on dst_device
 * (device pointers; a copy-engine transfer enqueued on `stream`, which must
 * belong to the current device).  The reference keeps one replica of the
 * filter words per NUMA node, made on first use by a thread of that node
 * (filter.hpp:128-152); the host mirror (dtlg.filter) keeps one per GPU the
 * same way and probes each device's keys against its own replica. */
dtlg_status dtlg_copy_words_peer(uint64_t* dst, int dst_device, const uint64_t* src, int src_device,
                                 uint64_t n_words, dtlg_stream_t stream);

/* ---- the L2 gather roofline (measurement; no reference counterpart) ----
 * Gathers n_sectors random 32-byte sectors of buf[0, bytes) (a device
 * pointer, 32-byte aligned) with the probe kernels' 256-bit read-only load
 * and XORs every word into *sink_dev (mixed, so the loads cannot be dropped).
 * Sector i is row ((h(i) mod 2^32) * (bytes / 32)) >> 32 of the buffer, h a
 * 64-bit multiply-xorshift hash of i + 1.  Timed over a buffer the size of an
 * L2-resident filter, it gives the rate that bounds that filter's probe. */
dtlg_status dtlg_sector_gather(const uint64_t* buf, uint64_t bytes, uint64_t n_sectors, uint64_t* sink_dev,
                               dtlg_stream_t stream);

/* ---- failure detection of the device waits (no reference counterpart) ----
 * The look-back of the ordered compaction and the batched kernel's item
 * dependencies wait on words written by other CTAs, each wait bounded; one
 * that runs out sets an error bit and the call reports DTLG_ERR_TIMEOUT.
 * This runs both wait loops on the current device against words that nothing
 * ever sets, with `spin_limit` spins (1 .. 2^22; each spin sleeps ~0.1 us),
 * synchronizes the device and stores the error bits they set in *err_bits:
 * bit 0 the look-back, bit 1 the dependency wait (3 = both gave up and
 * reported; the kernel ends either way and the context stays usable). */
dtlg_status dtlg_check_wait_timeout(uint32_t spin_limit, uint32_t* err_bits);

/* ---- single keys: filter_base::insert / contains (filter_base.hpp:22,32) ---- */
dtlg_status dtlg_insert(const dtlg_filter* f, uint64_t* filter_words, uint32_t key, dtlg_stream_t stream);
dtlg_status dtlg_contains(const dtlg_filter* f, const uint64_t* filter_words, uint32_t key,
                          int* result, dtlg_stream_t stream);

/* ---- host-buffer forms (the reference's calling convention: all host memory).
 * Keys and positions are HOST pointers; the filter words stay on the device.
 * Copies are staged through pinned memory in chunks that overlap the kernels. */
dtlg_status dtlg_batch_contains_host(const dtlg_filter* f, const uint64_t* filter_words,
                                     const uint32_t* keys_host, uint64_t key_cnt,
                                     uint32_t* match_positions_host, uint32_t match_offset,
                                     uint64_t* match_cnt, dtlg_stream_t stream);
dtlg_status dtlg_batch_insert_host(const dtlg_filter* f, uint64_t* filter_words,
                                   const uint32_t* keys_host, uint64_t key_cnt, uint64_t* failed_out,
                                   dtlg_stream_t stream);

/* ---- cuckoo helpers (cuckoofilter_logic.hpp:496-504) ---- */
dtlg_status dtlg_count_occupied_slots(const dtlg_filter* f, const uint64_t* filter_words,
                                      uint64_t* count, dtlg_stream_t stream);

/* ---- library ---- */
const char* dtlg_status_string(dtlg_status s);
const char* dtlg_last_cuda_error(void);
const char* dtlg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DTLG_H */
