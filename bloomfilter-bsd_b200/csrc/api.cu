// api.cu -- the C ABI of libdtlg.so (include/dtlg.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dtlg.h"
#include "filter_handle.hpp"
#include "host_config.hpp"
#include "registry.hpp"

using namespace dtlg;

namespace dtlg {

// ---- registry ----------------------------------------------------------------
static std::vector<BloomKernels>& bloom_table() {
  static std::vector<BloomKernels> t;
  return t;
}
static std::vector<CuckooKernels>& cuckoo_table() {
  static std::vector<CuckooKernels> t;
  return t;
}
static std::vector<BcfKernels>& bcf_table() {
  static std::vector<BcfKernels> t;
  return t;
}
void register_bloom(const BloomKernels& k) { bloom_table().push_back(k); }
void register_cuckoo(const CuckooKernels& k) { cuckoo_table().push_back(k); }
void register_bcf(const BcfKernels& k) { bcf_table().push_back(k); }
static std::vector<ClassicKernels>& classic_table() {
  static std::vector<ClassicKernels> t;
  return t;
}
void register_classic(const ClassicKernels& k) { classic_table().push_back(k); }
const ClassicKernels* find_classic() { return classic_table().empty() ? nullptr : &classic_table()[0]; }
const BcfKernels* find_bcf(uint32_t t, uint32_t a) {
  for (const auto& e : bcf_table())
    if (e.t == t && e.a == a) return &e;
  return nullptr;
}
const BloomKernels* find_bloom(uint32_t wb, uint32_t w, uint32_t s, uint32_t z, uint32_t k) {
  for (const auto& e : bloom_table())
    if (e.word_bytes == wb && e.w == w && e.s == s && e.z == z && e.k == k) return &e;
  return nullptr;
}
const CuckooKernels* find_cuckoo(uint32_t t, uint32_t b) {
  for (const auto& e : cuckoo_table())
    if (e.t == t && e.b == b) return &e;
  return nullptr;
}
int registered_bloom_count() { return static_cast<int>(bloom_table().size()); }

// ---- per-device state ----------------------------------------------------------
namespace {
thread_local std::string g_last_cuda_error;

struct DeviceState {
  bool init = false;
  int sms = 0;
  cudaMemPool_t pool = nullptr;
};
std::mutex g_mu;
DeviceState g_dev[64];

dtlg_status cuda_fail(cudaError_t e) {
  g_last_cuda_error = cudaGetErrorString(e);
  return DTLG_ERR_CUDA;
}

#define DTLG_CUDA(x)                         \
  do {                                       \
    cudaError_t _e = (x);                    \
    if (_e != cudaSuccess) return cuda_fail(_e); \
  } while (0)

dtlg_status device_state(DeviceState** out) {
  int dev = 0;
  DTLG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return DTLG_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState& s = g_dev[dev];
  if (!s.init) {
    DTLG_CUDA(cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev));
    // A library-private stream-ordered pool for per-call workspaces; it keeps
    // its memory between calls instead of returning it at every sync.
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    DTLG_CUDA(cudaMemPoolCreate(&s.pool, &props));
    uint64_t thr = ~0ull;
    DTLG_CUDA(cudaMemPoolSetAttribute(s.pool, cudaMemPoolAttrReleaseThreshold, &thr));
    s.init = true;
  }
  *out = &s;
  return DTLG_OK;
}

// Workspace of one probe call: header (tile counter, error word, count) then
// one look-back status word per tile.
struct WsHeader {
  unsigned int tile_ctr;
  unsigned int err;
  unsigned long long count;
  unsigned long long pad[14];
};
static_assert(sizeof(WsHeader) == 128, "header is one 128-byte line");

uint32_t probe_tiles(uint64_t n_phys) { return static_cast<uint32_t>((n_phys + kProbeTile - 1) / kProbeTile); }

// Two-pass layout inside the same workspace: header | status words | bitmask.
constexpr uint64_t kTwoPassMinKeys = 1ull << 20;
uint64_t bits_words(uint64_t n_phys) { return (n_phys + 31) / 32; }
uint32_t compact_tiles(uint64_t n_phys) {
  return static_cast<uint32_t>((bits_words(n_phys) + kCompactTileWords - 1) / kCompactTileWords);
}
size_t status_bytes(uint64_t n_phys) {
  const uint64_t t = std::max<uint64_t>(probe_tiles(n_phys), compact_tiles(n_phys));
  return static_cast<size_t>(((t * 8 + 255) / 256) * 256);
}
size_t round256(uint64_t b) { return static_cast<size_t>(((b + 255) / 256) * 256); }
uint32_t part_tiles(uint64_t n_phys) { return static_cast<uint32_t>((n_phys + kPartTile - 1) / kPartTile); }

// Workspace: header | status words | match bitmask | [partitioned probe:
// partition header (range fill counters) | per-tile overflow masks |
// (key, position) pairs in one segment per range]
struct WsLayout {
  size_t bits_off, part_off, tflags_off, pairs_off, total_small, total;
};
WsLayout ws_layout(uint64_t n_phys) {
  WsLayout l{};
  l.bits_off = sizeof(WsHeader) + status_bytes(n_phys);
  l.part_off = l.bits_off + round256(bits_words(n_phys) * 4);
  l.total_small = l.part_off;
  l.tflags_off = l.part_off + kPartHeaderBytes;
  l.pairs_off = l.tflags_off + round256(static_cast<uint64_t>(part_tiles(n_phys)) * 8);
  l.total = l.pairs_off + round256(part_pair_capacity(n_phys) * 8 + 16);
  return l;
}
size_t workspace_bytes(uint64_t n_phys) { return ws_layout(n_phys).total; }

int compact_occupancy() {
  static int occ = [] {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, compact_kernel, kCompactThreads, 0);
    return std::max(1, n);
  }();
  return occ;
}

// Block-range passes of the two-pass probe.  Random probes over more than
// ~256 MiB of filter run out of the GPU's address-translation reach (B200: the
// probe rate falls from ~62 to ~25 Gkeys/s between 256 and 512 MiB), so larger
// filters are probed in passes of about 256 MiB each; filters up to 160 MiB
// take one pass.  dtlg_set_probe_passes overrides the choice.
uint32_t probe_passes(const dtlg_filter* f) {
  // a classic Bloom key's k words lie anywhere in the filter, and a key
  // matches only if all are set: its probe cannot be split by word range
  if (f->qk) return 1;
  const uint64_t bytes = (f->d.m_actual + 7) / 8;
  uint64_t r = f->probe_passes;
  if (r == 0 && f->ck) {
    // Cuckoo buckets are 1-16 bytes but an L2 miss fills 64 bytes, so a table
    // beyond L2 wastes most of its DRAM traffic: probe it in passes whose
    // bucket range (<= 72 MiB) stays in the 126 MB L2.  B200, t=16 b=4,
    // 141 MB table, 2^28 probes: 1 pass 52.3, 2 passes 81.4, 3 passes 64.9 Gkeys/s.
    r = bytes <= (64ull << 20) ? 1 : (bytes + (72ull << 20) - 1) / (72ull << 20);
  } else if (r == 0) {
    r = bytes <= (160ull << 20) ? 1 : std::max<uint64_t>(2, (bytes + (128ull << 20)) / (256ull << 20));
  }
  r = std::min<uint64_t>(r, 16);
  r = std::min<uint64_t>(r, std::max<uint32_t>(1, f->d.addr.block_cnt));
  return static_cast<uint32_t>(std::max<uint64_t>(1, r));
}

dtlg_status check_filter_ptr(const void* p) {
  if (!p) return DTLG_ERR_NULL;
  if (reinterpret_cast<uintptr_t>(p) & 15u) return DTLG_ERR_ALIGNMENT;
  return DTLG_OK;
}

// Probe kernel plan for n keys: 1 = fused (probe + ordered compaction in one
// kernel), 2 = match bitmask in block-range passes + compaction,
// 3 = partitioned probe (Bloom and blocked cuckoo filters: one block per key)
// + compaction, 4 = match bitmask against a shared-memory copy of a filter of
// at most kSmemMaxBytes (Bloom and classic Bloom filters) + compaction.
// Automatic choice (measured on B200, u64 w=8 s=8 k=8, 2^26-2^28 probes):
// below 2^20 keys the single fused kernel; Bloom filters above 160 MiB the
// partitioned probe (256 MiB: 68.6 vs 62.5 Gkeys/s; 512 MiB: 64 vs 54); else
// the bitmask kernel (L2-resident filters: 113 vs 76 Gkeys/s partitioned).
// Plan 4 is offered up to kSmemMaxBytes (below every sm_100 opt-in limit,
// 227 KiB) but never chosen automatically: on B200 a small filter read through
// L1 probes faster than a shared-memory copy (64 KiB u64 w=8 s=8 k=8 filter,
// 2^28 probes: 141.5 Gkeys/s plan 2, 101.5 plan 4 -- random 16-byte shared
// loads conflict on banks, L1 hits do not).  The autotuner times it.
constexpr uint64_t kSmemMaxBytes = 192ull << 10;
// Filters larger than this take the L1 no-allocate loads in plan 2 (B200,
// u64 w=8 s=8 k=8, 2^28 probes, allocating: 128 KiB 155, 256 KiB 126, 512 KiB
// 112 Gkeys/s; not allocating, 1-8 MiB: 128.7).
constexpr uint64_t kL1NoAllocBytes = 256ull << 10;

// Blocked Bloom filters just beyond the single-pass limit whose words the
// hash picks one by one (s < w), or of one word per block, and zoned u32
// filters of 192 MiB: the bitmask plan in its block-range passes with the
// 32-register variant beats the partitioned plan.  B200, 2^27 probes, Gkeys/s,
// bitmask vs partition:
//   u32 w=16 s=1 k=4    192 / 224 / 256 MiB: 106.1 / 98.1 / 90.4 vs 81.9 / 82.9 / 83.3
//   u64 w=8 s=2 k=8     192 MiB: 75.9 vs 64.0
//   u32 w=1 k=4         168 / 192 MiB: 136.2 / 119.5 vs 102.7 / 104.1 (256: 93.6 vs 105.9)
//   zoned u32 w=16 z=2  192 / 256 MiB: 105.0 / 89.6 vs 97.9 / 100.6
// Layouts that test half a block before loading the rest (s >= w with blocks
// of >= 64 bytes) and zoned u64 ones probe faster partitioned from 160 MiB on
// (u64 w=8 s=8 k=8 168 / 192 MiB: 89.8 / 85.5 vs 91.2 / 88.9; zoned u64 w=8
// z=4 192 MiB: 74.6 vs 83.9; z=2 256 MiB: 87.8 vs 94.4), as do 32-byte blocks
// (u64 w=4 s=4 k=8, 168 MiB: 83.9 vs 89.7).
bool bitmask_band(const dtlg_filter* f) {
  if (f->d.kind != Kind::kBloom && f->d.kind != Kind::kZoned) return false;
  const uint64_t fbytes = (f->d.m_actual + 7) / 8;
  const uint64_t block_bytes = static_cast<uint64_t>(f->d.w) * f->d.word_bytes;
  if (fbytes <= (160ull << 20)) return false;
  // the limits leave room for MAGIC sizes, which round a request up
  if (f->d.kind == Kind::kZoned) return f->d.word_bytes == 4 && fbytes <= (224ull << 20);
  if (f->d.s < f->d.w) return fbytes <= (264ull << 20);
  return block_bytes < 32 && fbytes <= (240ull << 20);
}

int probe_plan(const dtlg_filter* f, uint64_t n) {
  int mode = f->probe_mode;
  const bool partitioned = f->pk->probe_pairs[0] != nullptr;
  const uint64_t fbytes = (f->d.m_actual + 7) / 8;
  const bool smem = f->pk->probe_smem != nullptr && fbytes <= kSmemMaxBytes;
  if (mode == 3 && !partitioned) mode = 2;
  if (mode == 4 && !smem) mode = 2;
  if (mode == 0) {
    if (n < kTwoPassMinKeys) {
      mode = 1;
    } else if (bitmask_band(f)) {
      mode = 2;
    } else {
      mode = (partitioned && fbytes > (160ull << 20)) ? 3 : 2;
    }
  }
  return mode;
}

// Register-budget variant of the bitmask / pair kernels for plan `mode`: the
// caller's, else 0 for the bitmask plan in the band above and for the pair
// probe of Bloom filters, else 1.  Pair probe, v0 against v1, Gkeys/s:
// u64 w=8 s=8 k=8 at 192 / 256 / 512 MiB 88.9 / 91.5 / 84.9 against 84.8 /
// 85.3 / 80.4 with 32 MiB ranges, 92.2 / 94.3 / 89.0 against 89.7 / 92.1 /
// 90.5 with 8 MiB ranges; zoned u64 w=8 z=2 at 256 / 384 MiB 94.4 / 91.1
// against 92.7 / 88.3.
// A 32-register bitmask kernel that spills (local memory per thread, from
// cudaFuncGetAttributes; -Xptxas -v: 19 layouts) gives way to the 64-register
// one: u64 w=1 k=16 at 200 MiB, 2^27 probes, spilling v0 65.1 against v1 69.3
// Gkeys/s.  The pair probe keeps v0 where it spills (7 layouts, all k >= 12):
// its spills cost less than the halved occupancy of v1 (u64 w=8 s=8 k=16 at
// 512 MiB: 83.0 against 79.7; u64 w=4 s=4 k=16 at 192 MiB: 89.7 against 87.5).
int probe_variant(const dtlg_filter* f, int mode) {
  if (f->bits_variant >= 0 && f->bits_variant < kBitsVariants) return f->bits_variant;
  if (mode == 3) return (f->d.kind == Kind::kBloom || f->d.kind == Kind::kZoned) ? 0 : 1;
  int v = bitmask_band(f) ? 0 : 1;
  if (v == 0) {
    const occ_fn spill = f->pk->bits_local_bytes[0];
    if (spill && spill() != 0) v = 1;
  }
  return v;
}

// Ranges of the partitioned probe and build: 2^L blocks each, about 8 MiB of
// filter and at most kMaxRanges of them.  A range shares L2 with the pair
// stream and the match mask's atomics; smaller ranges are re-read less (B200,
// u64 w=8 s=8 k=8, 2^28 probes, 32 / 16 / 8 MiB ranges: 512 MiB filter 85.8 /
// 87.2 / 89.9 Gkeys/s, 256 MiB 94.8 / 97.0 / 96.2; 512 MiB build from 2^28
// keys 19.9 / 19.0 / 18.5 ms).
void partition_ranges(const dtlg_filter* f, uint32_t* range_log2, uint32_t* n_ranges) {
  const uint64_t block_bytes = static_cast<uint64_t>(f->d.w) * f->d.word_bytes;
  const uint64_t nb = f->d.addr.block_cnt;
  uint32_t L = 0;
  while ((1ull << L) * block_bytes < (8ull << 20) && (1ull << L) < nb) L++;
  while (((nb + (1ull << L) - 1) >> L) > static_cast<uint64_t>(kMaxRanges)) L++;
  *range_log2 = L;
  *n_ranges = static_cast<uint32_t>((nb + (1ull << L) - 1) >> L);
}

// Groups keys_al[pre, n_phys) by filter range: (key, logical position) pairs
// in one segment per range, in the workspace's pair area (partitioned probe
// and build).  The partition header must be zeroed before (it is, with the
// match mask, by one memset).  One kernel, grids of resident CTAs only: the
// tiles are strided over the grid, so a second, partial wave would finish its
// share late.  spill: optional exact list of the pairs that did not fit.
cudaError_t launch_partition(const dtlg_filter* f, const uint32_t* keys_al, uint64_t n_phys, uint32_t pre,
                             char* wsb, const WsLayout& lay, int sms, cudaStream_t stream, PartArgs* out,
                             uint2* spill = nullptr) {
  PartArgs pa{};
  pa.keys_al = keys_al;
  pa.n_phys = n_phys;
  pa.pre = pre;
  pa.addr = f->d.addr;
  pa.block_mul = mul_const(f->xk ? 1 : 0);
  partition_ranges(f, &pa.range_log2, &pa.n_ranges);
  pa.n_tiles = part_tiles(n_phys);
  part_segments(n_phys - pre, f->d.addr.block_cnt, pa.range_log2, pa.n_ranges, &pa.seg_cap, &pa.last_cap);
  pa.hdr = reinterpret_cast<PartHeader*>(wsb + lay.part_off);
  pa.tile_overflow = reinterpret_cast<unsigned long long*>(wsb + lay.tflags_off);
  pa.pairs = reinterpret_cast<uint2*>(wsb + lay.pairs_off);
  pa.spill = spill;
  auto occupancy = [](void (*k)(PartArgs)) {
    int o = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k, kPartThreads, 0) == cudaSuccess ? std::max(1, o) : 1;
  };
  static const int occ_pow2 = occupancy(part_scatter_kernel<false>);
  static const int occ_magic = occupancy(part_scatter_kernel<true>);
  const bool magic = pa.addr.magic_mode != 0;
  const int sgrid = static_cast<int>(
      std::min<uint64_t>(pa.n_tiles, static_cast<uint64_t>(sms) * (magic ? occ_magic : occ_pow2)));
  if (magic) {
    part_scatter_kernel<true><<<sgrid, kPartThreads, 0, stream>>>(pa);
  } else {
    part_scatter_kernel<false><<<sgrid, kPartThreads, 0, stream>>>(pa);
  }
  *out = pa;
  return cudaGetLastError();
}

// Payload columns copied along with the match positions (probe -> gather).
struct GatherSpec {
  uint32_t n_cols;
  uint32_t col_bytes[kMaxGatherCols];
  const void* cols[kMaxGatherCols];
  void* out_cols[kMaxGatherCols];
};

// Enqueues the probe of `keys[0..n)`; the count goes to count_dev.  With
// `gather`, the compaction also copies the matching rows of the payload
// columns (the fused single-kernel plan has no compaction pass of its own,
// so gathers always take the bitmask plan).
dtlg_status launch_probe(const dtlg_filter* f, const uint64_t* words, const uint32_t* keys, uint32_t n,
                         uint32_t* out, uint32_t offset, unsigned long long* count_dev, void* ws,
                         size_t ws_bytes, cudaStream_t stream, const GatherSpec* gather = nullptr) {
  DeviceState* ds = nullptr;
  dtlg_status st = device_state(&ds);
  if (st) return st;
  if (n == 0) {
    DTLG_CUDA(cudaMemsetAsync(count_dev, 0, sizeof(unsigned long long), stream));
    return DTLG_OK;
  }
  const uint32_t pre = static_cast<uint32_t>((reinterpret_cast<uintptr_t>(keys) & 15u) >> 2);
  const uint64_t n_phys = static_cast<uint64_t>(n) + pre;
  int mode = probe_plan(f, n);
  if (gather && mode == 1) mode = 2;
  const uint32_t tiles = mode == 1 ? probe_tiles(n_phys) : compact_tiles(n_phys);
  const WsLayout lay = ws_layout(n_phys);
  if (ws_bytes < (mode == 3 ? lay.total : lay.total_small)) return DTLG_ERR_WORKSPACE;
  DTLG_CUDA(cudaMemsetAsync(ws, 0, sizeof(WsHeader) + static_cast<size_t>(tiles) * 8, stream));
  char* wsb = static_cast<char*>(ws);
  WsHeader* h = static_cast<WsHeader*>(ws);
  ProbeArgs a{};
  a.filter = words;
  a.keys_al = keys - pre;
  a.n_phys = n_phys;
  a.pre = pre;
  a.match_offset = offset;
  a.out = out;
  a.count_out = count_dev;
  a.status = reinterpret_cast<unsigned long long*>(h + 1);
  a.tile_ctr = &h->tile_ctr;
  a.err = &h->err;
  a.n_tiles = tiles;
  set_filter_args(f->d, &a);
  // blocks of >= 32 bytes are read with 256-bit loads when the words are
  // 32-byte aligned (every plan; the fused plan read them as two 128-bit
  // loads before, which doubled its L1 wavefronts)
  a.vec32 = (reinterpret_cast<uintptr_t>(words) & 31u) == 0 ? 1u : 0u;
  if (mode == 1) {
    // the fused plan reads Bloom filters that cannot live in L1 without
    // allocating there, as the bitmask plan does (below)
    a.l1na = (f->bk != nullptr && (f->d.m_actual / 8) > kL1NoAllocBytes) ? 1u : 0u;
    const probe_fn fn = f->pk->probe;
    const occ_fn occ = f->pk->probe_blocks_per_sm;
    const int per_sm = std::max(1, occ());
    const int grid = static_cast<int>(std::min<uint64_t>(tiles, static_cast<uint64_t>(ds->sms) * per_sm));
    DTLG_CUDA(fn(a, grid, stream));
    return DTLG_OK;
  }
  uint32_t* bits = reinterpret_cast<uint32_t*>(wsb + lay.bits_off);
  const int v = probe_variant(f, mode);
  if (mode == 4) {
    // the whole filter in every CTA's shared memory
    const uint32_t words32 = static_cast<uint32_t>((f->d.m_actual + 31) / 32);
    DTLG_CUDA(f->pk->probe_smem(a, bits, words32, (n_phys + 127) / 128, ds->sms, stream));
  } else if (mode == 2) {
    // Random blocks of a Bloom filter that cannot live in L1 are read without
    // allocating in L1 (B200, u64 w=8 s=8 k=8, 2^28 probes: 8 MiB filter
    // 118.5 -> 127.1 Gkeys/s; a 64 KiB L1-resident filter falls from 150.8 to
    // 71.1 without L1 allocation, and the partitioned plan's pair probe from
    // 76.0 to 72.9, so both keep allocating).  Not for the other kinds:
    // cuckoo buckets 75.6 -> 47.9, blocked cuckoo (128 MiB) 102.1 -> 98.9,
    // classic Bloom unchanged.
    a.l1na = (f->bk != nullptr && (f->d.m_actual / 8) > kL1NoAllocBytes) ? 1u : 0u;
    // match bitmask, in block-range passes over large filters (each pass
    // probes only the keys whose block lies in its range, so the concurrently
    // touched part of the filter stays within the GPU's address-translation reach)
    const probe_bits_fn bfn = f->pk->probe_bits[v];
    const occ_fn bocc = f->pk->bits_blocks_per_sm[v];
    const uint64_t chunks = (n_phys + 127) / 128;  // one warp-chunk = 128 keys
    const uint64_t max_grid = static_cast<uint64_t>(ds->sms) * std::max(1, bocc());
    const int bgrid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((chunks + 7) / 8, max_grid)));
    const uint32_t passes = probe_passes(f);
    const uint32_t nb = f->d.addr.block_cnt;
    for (uint32_t r = 0; r < passes; r++) {
      a.range_on = passes > 1 ? 1u : 0u;
      a.blk_lo = static_cast<uint32_t>(static_cast<uint64_t>(nb) * r / passes);
      a.blk_hi = r + 1 == passes ? 0xFFFFFFFFu : static_cast<uint32_t>(static_cast<uint64_t>(nb) * (r + 1) / passes);
      DTLG_CUDA(bfn(a, bits, r > 0 ? 1 : 0, bgrid, stream));
    }
  } else {
    // partitioned probe: keys grouped by filter range, probed range by range;
    // one memset zeroes the match mask and the partition header after it
    PartArgs pa{};
    DTLG_CUDA(cudaMemsetAsync(bits, 0, lay.part_off - lay.bits_off + kPartHeaderBytes, stream));
    DTLG_CUDA(launch_partition(f, a.keys_al, n_phys, pre, wsb, lay, ds->sms, stream, &pa));
    PairsArgs pr{};
    pr.probe = a;
    pr.part = pa;
    pr.bits = bits;
    pr.pre = pre;
    const int qgrid = static_cast<int>(static_cast<uint64_t>(ds->sms) * std::max(1, f->pk->pairs_blocks_per_sm[v]()));
    DTLG_CUDA(f->pk->probe_pairs[v](pr, qgrid, stream));
  }
  // ordered compaction of the bitmask
  CompactArgs c{};
  c.bits = bits;
  c.n_words = bits_words(n_phys);
  c.pre = pre;
  c.match_offset = offset;
  c.out = out;
  c.count_out = count_dev;
  c.status = a.status;
  c.tile_ctr = a.tile_ctr;
  c.err = a.err;
  c.n_tiles = tiles;
  if (gather) {
    c.n_cols = gather->n_cols;
    for (uint32_t i = 0; i < gather->n_cols; i++) {
      c.col_bytes[i] = gather->col_bytes[i];
      c.cols[i] = gather->cols[i];
      c.out_cols[i] = gather->out_cols[i];
    }
  }
  const int cgrid = static_cast<int>(std::min<uint64_t>(tiles, static_cast<uint64_t>(ds->sms) * compact_occupancy()));
  compact_kernel<<<cgrid, kCompactThreads, 0, stream>>>(c);
  DTLG_CUDA(cudaGetLastError());
  return DTLG_OK;
}

// Build plan of a blocked Bloom or blocked cuckoo filter (one block per key)
// for n keys: 1 = one kernel of global atomics, 2 = keys grouped by L2-sized
// block range first (the probe's partition).  Automatic: the partitioned
// build for Bloom filters beyond 80 MiB and batches of >= 2^20 keys (u64 w=8
// s=8 k=8, plan 1 -> plan 2: 512 MiB from 2^28 keys 10.55 -> 4.07 ms; 256 MiB
// 4.23 -> 2.07 ms; 96 MiB (12 bits/key, MAGIC) 1.22 -> 1.09 ms; 64 MiB stays
// with plan 1, 0.51 against 0.60 ms).  A blocked cuckoo key takes one or two
// compare-and-swaps, too few to repay the partition (256 MiB, 2^26 keys:
// 2.60 -> 2.70 ms), so its plan 2 is only taken on request.
int block_build_plan(const dtlg_filter* f, uint64_t n) {
  if (f->build_mode == 1 || f->build_mode == 2) return f->build_mode;
  const uint64_t bytes = (f->d.m_actual + 7) / 8;
  return (f->bk != nullptr && n >= kTwoPassMinKeys && bytes > (80ull << 20)) ? 2 : 1;
}

int grid_for(uint64_t items, int sms) {
  return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((items + 255) / 256, static_cast<uint64_t>(sms) * 8)));
}

dtlg_status cuckoo_insert(const dtlg_filter* f, uint64_t* words, const uint32_t* keys, uint32_t n,
                          uint64_t* failed_out, cudaStream_t stream) {
  DeviceState* ds = nullptr;
  dtlg_status st = device_state(&ds);
  if (st) return st;
  if (failed_out) *failed_out = 0;
  if (n == 0) return DTLG_OK;
  const FilterDesc& d = f->d;
  const uint64_t slots_n = (static_cast<uint64_t>(d.addr.block_cnt) + 1) * d.b;
  uint32_t* slots = nullptr;
  unsigned long long* failed = nullptr;
  const uint64_t slot_bytes = (slots_n * 4 + 255) & ~255ull;
  DTLG_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&slots), slot_bytes + 256, ds->pool, stream));
  failed = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(slots) + slot_bytes);
  DTLG_CUDA(cudaMemsetAsync(failed, 0, 8, stream));
  DTLG_CUDA(cudaMemsetAsync(slots + static_cast<uint64_t>(d.addr.block_cnt) * d.b, 0, d.b * 4, stream));
  uint32_t* table = reinterpret_cast<uint32_t*>(words);
  f->ck->unpack(table, slots, d.addr.block_cnt, grid_for(slots_n, ds->sms), stream);
  const uint32_t pre = static_cast<uint32_t>((reinterpret_cast<uintptr_t>(keys) & 15u) >> 2);
  CuckooBuildArgs a{};
  a.table = table;
  a.slots = slots;
  a.keys_al = keys - pre;
  a.n_phys = static_cast<uint64_t>(n) + pre;
  a.pre = pre;
  a.table_words = d.word_cnt;
  a.victim_word = d.victim_word;
  a.addr = d.addr;
  a.failed = failed;
  static std::atomic<uint64_t> seed_ctr{0x243F6A8885A308D3ull};
  a.seed = seed_ctr.fetch_add(0x9E3779B97F4A7C15ull);
  f->ck->insert(a, grid_for(a.n_phys, ds->sms), stream);
  f->ck->pack(table, slots, d.addr.block_cnt, d.word_cnt, grid_for(d.word_cnt, ds->sms), stream);
  unsigned long long lost = 0;
  DTLG_CUDA(cudaMemcpyAsync(&lost, failed, 8, cudaMemcpyDeviceToHost, stream));
  DTLG_CUDA(cudaFreeAsync(slots, stream));
  DTLG_CUDA(cudaStreamSynchronize(stream));
  DTLG_CUDA(cudaGetLastError());
  if (failed_out) *failed_out = lost;
  return lost ? DTLG_ERR_CUCKOO_FULL : DTLG_OK;
}

}  // namespace

dtlg_status cuda_error_status(cudaError_t e) { return cuda_fail(e); }
}  // namespace dtlg

// =============================================================================
extern "C" {

const char* dtlg_version(void) { return "dtlg 0.1 (sm_100a)"; }

const char* dtlg_last_cuda_error(void) { return dtlg::g_last_cuda_error.c_str(); }

const char* dtlg_status_string(dtlg_status s) {
  switch (s) {
    case DTLG_OK: return "ok";
    case DTLG_ERR_INVALID_CONFIG: return "invalid configuration";
    case DTLG_ERR_SIZE: return "filter size out of range (block count must not exceed 2^31)";
    case DTLG_ERR_NULL: return "null pointer";
    case DTLG_ERR_ALIGNMENT: return "filter words must be 16-byte aligned";
    case DTLG_ERR_CUDA: return "CUDA error";
    case DTLG_ERR_ALLOC: return "allocation failed";
    case DTLG_ERR_CUCKOO_FULL: return "cuckoo filter full: some keys could not be inserted";
    case DTLG_ERR_TIMEOUT: return "a bounded device wait timed out";
    case DTLG_ERR_WORKSPACE: return "workspace too small";
    case DTLG_ERR_UNSUPPORTED: return "unsupported operation";
  }
  return "unknown status";
}

dtlg_status dtlg_bloom_create(const dtlg_bloom_config* cfg, uint64_t m, dtlg_filter** out) {
  if (!cfg || !out) return DTLG_ERR_NULL;
  *out = nullptr;
  dtlg_filter* f = new dtlg_filter();
  const int rc = describe_bloom(cfg->word_size, cfg->word_cnt_per_block, cfg->sector_cnt, cfg->zone_cnt,
                                cfg->k, m, &f->d);
  if (rc) {
    delete f;
    return rc == 1 ? DTLG_ERR_INVALID_CONFIG : DTLG_ERR_SIZE;
  }
  f->bk = find_bloom(f->d.word_bytes, f->d.w, f->d.s, f->d.z, f->d.k);
  if (!f->bk) {
    delete f;
    return DTLG_ERR_INVALID_CONFIG;
  }
  f->pk = &f->bk->pk;
  *out = f;
  return DTLG_OK;
}

dtlg_status dtlg_cuckoo_create(const dtlg_cuckoo_config* cfg, uint64_t m, dtlg_filter** out) {
  if (!cfg || !out) return DTLG_ERR_NULL;
  *out = nullptr;
  dtlg_filter* f = new dtlg_filter();
  const int rc = describe_cuckoo(cfg->bits_per_tag, cfg->tags_per_bucket, m, &f->d);
  if (rc) {
    delete f;
    return rc == 1 ? DTLG_ERR_INVALID_CONFIG : DTLG_ERR_SIZE;
  }
  f->ck = find_cuckoo(f->d.t, f->d.b);
  if (!f->ck) {
    delete f;
    return DTLG_ERR_INVALID_CONFIG;
  }
  f->pk = &f->ck->pk;
  *out = f;
  return DTLG_OK;
}

dtlg_status dtlg_classic_bloom_create(const dtlg_classic_bloom_config* cfg, uint64_t m, dtlg_filter** out) {
  if (!cfg || !out) return DTLG_ERR_NULL;
  *out = nullptr;
  if (cfg->addr_mode > 1) return DTLG_ERR_INVALID_CONFIG;
  dtlg_filter* f = new dtlg_filter();
  const int rc = describe_classic(cfg->k, m, cfg->addr_mode == 1, &f->d);
  if (rc) {
    delete f;
    return rc == 1 ? DTLG_ERR_INVALID_CONFIG : DTLG_ERR_SIZE;
  }
  f->qk = find_classic();
  if (!f->qk) {
    delete f;
    return DTLG_ERR_INVALID_CONFIG;
  }
  f->pk = &f->qk->pk;
  *out = f;
  return DTLG_OK;
}

dtlg_status dtlg_blocked_cuckoo_create(const dtlg_blocked_cuckoo_config* cfg, uint64_t m, dtlg_filter** out) {
  if (!cfg || !out) return DTLG_ERR_NULL;
  *out = nullptr;
  dtlg_filter* f = new dtlg_filter();
  const int rc = describe_bcf(cfg->block_size_bytes, cfg->tag_size_bits, cfg->associativity, m, &f->d);
  if (rc) {
    delete f;
    return rc == 1 ? DTLG_ERR_INVALID_CONFIG : DTLG_ERR_SIZE;
  }
  f->xk = find_bcf(f->d.t, f->d.b);
  if (!f->xk) {
    delete f;
    return DTLG_ERR_INVALID_CONFIG;
  }
  f->pk = &f->xk->pk;
  *out = f;
  return DTLG_OK;
}

void dtlg_destroy(dtlg_filter* f) { delete f; }

uint64_t dtlg_size_in_bytes(const dtlg_filter* f) { return f ? (f->d.m_actual + 7) / 8 : 0; }
uint64_t dtlg_size(const dtlg_filter* f) { return f ? f->d.size_u64 : 0; }
uint64_t dtlg_alloc_words_u64(const dtlg_filter* f) { return f ? f->d.alloc_u64 : 0; }
int dtlg_kind(const dtlg_filter* f) { return f ? static_cast<int>(f->d.kind) : -1; }
uint64_t dtlg_block_cnt(const dtlg_filter* f) { return f ? f->d.addr.block_cnt : 0; }
int dtlg_is_magic(const dtlg_filter* f) { return f ? static_cast<int>(f->d.addr.magic_mode) : 0; }

size_t dtlg_name(const dtlg_filter* f, char* buf, size_t cap) {
  if (!f) return 0;
  const std::string s = filter_name(f->d);
  if (buf && cap > s.size()) {
    std::memcpy(buf, s.c_str(), s.size() + 1);
  } else if (buf && cap) {
    buf[0] = 0;
  }
  return s.size();
}

dtlg_status dtlg_batch_insert(const dtlg_filter* f, uint64_t* words, const uint32_t* keys, uint32_t n,
                              uint64_t* failed_out, dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!f) return DTLG_ERR_NULL;
  if (failed_out) *failed_out = 0;
  if (n && !keys) return DTLG_ERR_NULL;
  if (dtlg_status st = check_filter_ptr(words)) return st;
  if (f->ck) return cuckoo_insert(f, words, keys, n, failed_out, stream);
  if (n == 0) return DTLG_OK;
  DeviceState* ds = nullptr;
  if (dtlg_status st = device_state(&ds)) return st;
  const uint32_t pre = static_cast<uint32_t>((reinterpret_cast<uintptr_t>(keys) & 15u) >> 2);
  if (f->qk) {
    ClassicBuildArgs c{};
    c.filter = reinterpret_cast<uint32_t*>(words);
    c.keys_al = keys - pre;
    c.n_phys = static_cast<uint64_t>(n) + pre;
    c.pre = pre;
    c.addr = f->d.addr;
    c.k = f->d.k;
    c.bit_shift = f->d.bit_shift;
    c.bit_mask = f->d.bit_mask;
    DTLG_CUDA(f->qk->build(c, grid_for(c.n_phys, ds->sms), stream));
    return DTLG_OK;
  }
  if (f->xk) {
    // blocked cuckoo: inserts never fail (bcf.cpp:36-40)
    BcfBuildArgs b{};
    b.filter = words;
    b.keys_al = keys - pre;
    b.n_phys = static_cast<uint64_t>(n) + pre;
    b.pre = pre;
    b.addr = f->d.addr;
    b.bucket_bits = f->d.bucket_bits;
    b.hash_shift = f->d.hash_shift;
    static std::atomic<uint64_t> seed_ctr{0x13198A2E03707344ull};
    b.seed = seed_ctr.fetch_add(0x9E3779B97F4A7C15ull);
    if (block_build_plan(f, n) == 2) {
      // keys grouped by L2-sized block range first, as for Bloom filters; the
      // pairs that overflow their segment go to an exact spill list after the
      // workspace (a blocked cuckoo key must be inserted exactly once)
      const WsLayout lay = ws_layout(b.n_phys);
      void* ws = nullptr;
      if (cudaMallocFromPoolAsync(&ws, lay.total + round256(b.n_phys * 8), ds->pool, stream) == cudaSuccess) {
        PartArgs pa{};
        char* wsb = static_cast<char*>(ws);
        cudaError_t e = cudaMemsetAsync(wsb + lay.part_off, 0, kPartHeaderBytes, stream);
        if (e == cudaSuccess)
          e = launch_partition(f, b.keys_al, b.n_phys, pre, wsb, lay, ds->sms, stream, &pa,
                               reinterpret_cast<uint2*>(wsb + lay.total));
        if (e == cudaSuccess) e = f->xk->insert_pairs(b, pa, grid_for(n, ds->sms), stream);
        cudaFreeAsync(ws, stream);
        DTLG_CUDA(e);
        return DTLG_OK;
      }
      cudaGetLastError();  // no room for the partition: the one-kernel build
    }
    DTLG_CUDA(f->xk->insert(b, grid_for(b.n_phys, ds->sms), stream));
    return DTLG_OK;
  }
  const uint64_t n_phys = static_cast<uint64_t>(n) + pre;
  if (block_build_plan(f, n) == 2) {
    // keys grouped by L2-sized block range first (the probe's partition), then
    // inserted range by range: the atomic ORs hit lines that sit in L2
    const WsLayout lay = ws_layout(n_phys);
    void* ws = nullptr;
    if (cudaMallocFromPoolAsync(&ws, lay.total, ds->pool, stream) == cudaSuccess) {
      PartArgs pa{};
      char* wsb = static_cast<char*>(ws);
      cudaError_t e = cudaMemsetAsync(wsb + lay.part_off, 0, kPartHeaderBytes, stream);
      if (e == cudaSuccess) e = launch_partition(f, keys - pre, n_phys, pre, wsb, lay, ds->sms, stream, &pa);
      if (e == cudaSuccess) {
        const uint64_t vec = (static_cast<uint64_t>(n) + 1) / 2;
        e = f->bk->build_pairs(pa, words, f->d.addr, grid_for(vec, ds->sms), stream);
      }
      cudaFreeAsync(ws, stream);
      DTLG_CUDA(e);
      return DTLG_OK;
    }
    // no room for the partition's 8 bytes per key: the one-kernel build
    // needs no workspace (same words)
    cudaGetLastError();
  }
  BuildArgs a{};
  a.filter = words;
  a.keys_al = keys - pre;
  a.n_phys = n_phys;
  a.pre = pre;
  a.addr = f->d.addr;
  DTLG_CUDA(f->bk->build(a, grid_for((a.n_phys + 3) / 4, ds->sms), stream));
  return DTLG_OK;
}

dtlg_status dtlg_set_build_options(dtlg_filter* f, int mode) {
  if (!f) return DTLG_ERR_NULL;
  if (mode < 0 || mode > 2) return DTLG_ERR_INVALID_CONFIG;
  f->build_mode = mode;
  return DTLG_OK;
}

size_t dtlg_probe_workspace_size(uint32_t key_cnt) { return workspace_bytes(static_cast<uint64_t>(key_cnt) + 3); }

dtlg_status dtlg_set_l2_fetch_granularity(int bytes, int* in_effect) {
  if (!(bytes == 0 || bytes == 32 || bytes == 64 || bytes == 128)) return DTLG_ERR_INVALID_CONFIG;
  DTLG_CUDA(cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, static_cast<size_t>(bytes)));
  size_t v = 0;
  DTLG_CUDA(cudaDeviceGetLimit(&v, cudaLimitMaxL2FetchGranularity));
  if (in_effect) *in_effect = static_cast<int>(v);
  return DTLG_OK;
}

int dtlg_probe_kernel_count(const dtlg_filter* f, uint32_t key_cnt) {
  if (!f || key_cnt == 0) return 0;
  const int mode = probe_plan(f, key_cnt);
  // plan 3: partition scatter, pair probe, overflow keys, compaction
  return mode == 1 ? 1 : (mode == 2 ? static_cast<int>(probe_passes(f)) + 1 : (mode == 4 ? 2 : 4));
}

dtlg_status dtlg_set_probe_passes(dtlg_filter* f, int passes) {
  if (!f) return DTLG_ERR_NULL;
  if (passes < 0 || passes > 16) return DTLG_ERR_INVALID_CONFIG;
  f->probe_passes = passes;
  return DTLG_OK;
}

dtlg_status dtlg_set_probe_options(dtlg_filter* f, int mode, int variant) {
  if (!f) return DTLG_ERR_NULL;
  if (mode < 0 || mode > 4 || variant < -1 || variant >= kBitsVariants) return DTLG_ERR_INVALID_CONFIG;
  f->probe_mode = mode;
  f->bits_variant = variant;
  return DTLG_OK;
}

dtlg_status dtlg_batch_contains_ws(const dtlg_filter* f, const uint64_t* words, const uint32_t* keys,
                                   uint32_t n, uint32_t* out, uint32_t offset, uint64_t* count_dev,
                                   void* ws, size_t ws_bytes, dtlg_stream_t stream) {
  if (!f || !count_dev || (n && (!keys || !out)) || !ws) return DTLG_ERR_NULL;
  if (dtlg_status st = check_filter_ptr(words)) return st;
  return launch_probe(f, words, keys, n, out, offset, reinterpret_cast<unsigned long long*>(count_dev), ws,
                      ws_bytes, reinterpret_cast<cudaStream_t>(stream));
}

dtlg_status dtlg_batch_contains_gather(const dtlg_filter* f, const uint64_t* words, const uint32_t* keys,
                                       uint32_t n, uint32_t n_cols, const void* const* cols,
                                       const uint32_t* col_bytes, void* const* out_cols, uint32_t* match_positions,
                                       uint32_t offset, uint64_t* count_dev, void* ws, size_t ws_bytes,
                                       dtlg_stream_t stream) {
  if (!f || !count_dev || !ws || (n && !keys)) return DTLG_ERR_NULL;
  if (n_cols > kMaxGatherCols || (n_cols == 0 && !match_positions)) return DTLG_ERR_INVALID_CONFIG;
  if (n_cols && (!cols || !col_bytes || !out_cols)) return DTLG_ERR_NULL;
  GatherSpec g{};
  g.n_cols = n_cols;
  for (uint32_t i = 0; i < n_cols; i++) {
    if (col_bytes[i] != 4 && col_bytes[i] != 8) return DTLG_ERR_INVALID_CONFIG;
    if (n && (!cols[i] || !out_cols[i])) return DTLG_ERR_NULL;
    g.col_bytes[i] = col_bytes[i];
    g.cols[i] = cols[i];
    g.out_cols[i] = out_cols[i];
  }
  if (dtlg_status st = check_filter_ptr(words)) return st;
  return launch_probe(f, words, keys, n, match_positions, offset, reinterpret_cast<unsigned long long*>(count_dev),
                      ws, ws_bytes, reinterpret_cast<cudaStream_t>(stream), &g);
}

dtlg_status dtlg_batch_contains_async(const dtlg_filter* f, const uint64_t* words, const uint32_t* keys,
                                      uint32_t n, uint32_t* out, uint32_t offset, uint64_t* count_dev,
                                      dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!f || !count_dev || (n && (!keys || !out))) return DTLG_ERR_NULL;
  if (dtlg_status st = check_filter_ptr(words)) return st;
  DeviceState* ds = nullptr;
  if (dtlg_status st = device_state(&ds)) return st;
  const size_t ws_bytes = dtlg_probe_workspace_size(n);
  void* ws = nullptr;
  DTLG_CUDA(cudaMallocFromPoolAsync(&ws, ws_bytes, ds->pool, stream));
  dtlg_status st = launch_probe(f, words, keys, n, out, offset, reinterpret_cast<unsigned long long*>(count_dev),
                                ws, ws_bytes, stream);
  cudaFreeAsync(ws, stream);
  return st;
}

dtlg_status dtlg_batch_contains(const dtlg_filter* f, const uint64_t* words, const uint32_t* keys, uint32_t n,
                                uint32_t* out, uint32_t offset, uint64_t* match_cnt, dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!f || !match_cnt || (n && (!keys || !out))) return DTLG_ERR_NULL;
  if (dtlg_status st = check_filter_ptr(words)) return st;
  DeviceState* ds = nullptr;
  if (dtlg_status st = device_state(&ds)) return st;
  const size_t ws_bytes = dtlg_probe_workspace_size(n);
  void* ws = nullptr;
  DTLG_CUDA(cudaMallocFromPoolAsync(&ws, ws_bytes, ds->pool, stream));
  WsHeader* h = static_cast<WsHeader*>(ws);
  dtlg_status st = launch_probe(f, words, keys, n, out, offset, &h->count, ws, ws_bytes, stream);
  WsHeader host{};
  if (st == DTLG_OK) {
    cudaError_t e = cudaMemcpyAsync(&host, h, 16, cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) st = cuda_fail(e);
  }
  cudaFreeAsync(ws, stream);
  if (st != DTLG_OK) return st;
  DTLG_CUDA(cudaStreamSynchronize(stream));
  if (n == 0) host.count = 0;
  *match_cnt = host.count;
  return host.err ? DTLG_ERR_TIMEOUT : DTLG_OK;
}

dtlg_status dtlg_insert(const dtlg_filter* f, uint64_t* words, uint32_t key, dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  DeviceState* ds = nullptr;
  if (dtlg_status st = device_state(&ds)) return st;
  uint32_t* k = nullptr;
  DTLG_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&k), 16, ds->pool, stream));
  DTLG_CUDA(cudaMemcpyAsync(k, &key, 4, cudaMemcpyHostToDevice, stream));
  dtlg_status st = dtlg_batch_insert(f, words, k, 1, nullptr, stream_);
  cudaFreeAsync(k, stream);
  DTLG_CUDA(cudaStreamSynchronize(stream));
  return st;
}

dtlg_status dtlg_contains(const dtlg_filter* f, const uint64_t* words, uint32_t key, int* result,
                          dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!result) return DTLG_ERR_NULL;
  DeviceState* ds = nullptr;
  if (dtlg_status st = device_state(&ds)) return st;
  uint32_t* k = nullptr;
  DTLG_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&k), 64, ds->pool, stream));
  DTLG_CUDA(cudaMemcpyAsync(k, &key, 4, cudaMemcpyHostToDevice, stream));
  uint64_t cnt = 0;
  dtlg_status st = dtlg_batch_contains(f, words, k, 1, k + 4, 0, &cnt, stream_);
  cudaFreeAsync(k, stream);
  DTLG_CUDA(cudaStreamSynchronize(stream));
  *result = cnt ? 1 : 0;
  return st;
}

dtlg_status dtlg_count_occupied_slots(const dtlg_filter* f, const uint64_t* words, uint64_t* count,
                                      dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!f || !count) return DTLG_ERR_NULL;
  if (!f->ck) return DTLG_ERR_UNSUPPORTED;
  if (dtlg_status st = check_filter_ptr(words)) return st;
  DeviceState* ds = nullptr;
  if (dtlg_status st = device_state(&ds)) return st;
  unsigned long long* c = nullptr;
  DTLG_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&c), 8, ds->pool, stream));
  DTLG_CUDA(cudaMemsetAsync(c, 0, 8, stream));
  const uint64_t slots = static_cast<uint64_t>(f->d.addr.block_cnt) * f->d.b;
  f->ck->count(reinterpret_cast<const uint32_t*>(words), f->d.addr.block_cnt, f->d.victim_word, c,
               grid_for(slots, ds->sms), stream);
  unsigned long long h = 0;
  DTLG_CUDA(cudaMemcpyAsync(&h, c, 8, cudaMemcpyDeviceToHost, stream));
  cudaFreeAsync(c, stream);
  DTLG_CUDA(cudaStreamSynchronize(stream));
  *count = h;
  return DTLG_OK;
}

}  // extern "C"
