// batched.cu -- host side of the batched multi-filter build+probe (batched.cuh).
//
// No counterpart in the reference: there a query with many filters calls
// filter_base::batch_insert and batch_contains once per filter
// (filter_base.hpp:26,42-45).  dtlg_batch_prepare turns a list of such calls
// into device tables once; dtlg_batch_run then executes all of them as one
// persistent kernel, captured with its workspace reset into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/dtlg.h"
#include "batched.cuh"
#include "filter_handle.hpp"

namespace {

using namespace dtlg;

// The configs compiled into the batched kernel: sectorized and zoned 64-byte
// blocks (u64 w=8 s=8; u64 w=8 z=2/4; u32 w=16 z=2/4, all k=8) and
// register-blocked u32 w=1 k=4/8.  Filters of any other config run as
// separate launches inside the same graph.
using Menu0 = BloomCfg<uint64_t, 8, 8, 1, 8>;
using Menu1 = BloomCfg<uint64_t, 8, 8, 2, 8>;
using Menu2 = BloomCfg<uint64_t, 8, 8, 4, 8>;
using Menu3 = BloomCfg<uint32_t, 16, 16, 2, 8>;
using Menu4 = BloomCfg<uint32_t, 16, 16, 4, 8>;
using Menu5 = BloomCfg<uint32_t, 1, 1, 1, 4>;
using Menu6 = BloomCfg<uint32_t, 1, 1, 1, 8>;
struct MenuEntry {
  uint32_t wb, w, s, z, k;
};
constexpr MenuEntry kMenu[] = {{8, 8, 8, 1, 8},   {8, 8, 8, 2, 8}, {8, 8, 8, 4, 8}, {4, 16, 16, 2, 8},
                               {4, 16, 16, 4, 8}, {4, 1, 1, 1, 4}, {4, 1, 1, 1, 8}};
constexpr auto kBatchedKernel = batched_kernel<Menu0, Menu1, Menu2, Menu3, Menu4, Menu5, Menu6>;

int menu_index(const FilterDesc& d) {
  if (d.kind != Kind::kBloom && d.kind != Kind::kZoned) return -1;
  for (int i = 0; i < static_cast<int>(sizeof(kMenu) / sizeof(kMenu[0])); i++) {
    const MenuEntry& m = kMenu[i];
    if (m.wb == d.word_bytes && m.w == d.w && m.s == d.s && m.z == d.z && m.k == d.k) return i;
  }
  return -1;
}

uint32_t tiles_of(uint32_t n) { return (n + kBatchTile - 1) / kBatchTile; }
size_t round256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

struct dtlg_batch {
  std::vector<dtlg_batch_item> items;
  std::vector<BatchDesc> desc;       // host copy (with staging as planned at prepare)
  uint32_t* d_bucket = nullptr;      // all staged filters' range buckets
  uint32_t* d_mask = nullptr;        // all filters' match bitmasks
  uint2* d_items[2] = {nullptr, nullptr};  // the queue with staged builds [0] / all direct [1]
  uint32_t n_items[2] = {0, 0};
  size_t ranges_built_off = 0, cursor_off = 0;
  int staging = 0;                   // 0: stage every filter that fits, 1: never
  std::vector<int> fallback;         // item indexes run as separate launches
  std::vector<void*> fallback_ws;
  std::vector<size_t> fallback_ws_bytes;
  uint32_t n_menu = 0, n_probe_tiles = 0, n_ctiles = 0;
  BatchDesc* d_desc = nullptr;
  char* d_ctl = nullptr;             // ctl words | built / ranges / probed counters | cursors | status words
  size_t ctl_bytes = 0, built_off = 0, probed_off = 0, status_off = 0;
  int sms = 0, occupancy = 1, ctas_per_sm = 0;
  bool use_graph = false;
  bool warm = false;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaStream_t cap = nullptr;
};

namespace {

dtlg_status enqueue(dtlg_batch* b, cudaStream_t s) {
  if (b->n_menu) {
    if (cudaMemsetAsync(b->d_ctl, 0, b->ctl_bytes, s) != cudaSuccess) return DTLG_ERR_CUDA;
    BatchArgs a{};
    a.desc = b->d_desc;
    a.n_filters = b->n_menu;
    a.ctl = reinterpret_cast<unsigned int*>(b->d_ctl);
    a.built = reinterpret_cast<unsigned int*>(b->d_ctl + b->built_off);
    a.ranges_built = reinterpret_cast<unsigned int*>(b->d_ctl + b->ranges_built_off);
    a.probed = reinterpret_cast<unsigned int*>(b->d_ctl + b->probed_off);
    a.items = b->d_items[b->staging == 1 ? 1 : 0];
    a.n_items = b->n_items[b->staging == 1 ? 1 : 0];
    a.status = reinterpret_cast<unsigned long long*>(b->d_ctl + b->status_off);
    const int per_sm = b->ctas_per_sm > 0 ? std::min(b->ctas_per_sm, b->occupancy) : b->occupancy;
    const uint32_t work = a.n_items;
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(work, static_cast<uint64_t>(b->sms) * per_sm)));
    kBatchedKernel<<<grid, kBatchThreads, kBatchRangeBytes, s>>>(a);
    if (cudaGetLastError() != cudaSuccess) return DTLG_ERR_CUDA;
  }
  for (size_t j = 0; j < b->fallback.size(); j++) {
    const dtlg_batch_item& it = b->items[b->fallback[j]];
    dtlg_stream_t ds = reinterpret_cast<dtlg_stream_t>(s);
    if (dtlg_status st = dtlg_batch_insert(it.filter, it.filter_words, it.build_keys, it.n_build, nullptr, ds)) return st;
    if (dtlg_status st = dtlg_batch_contains_ws(it.filter, it.filter_words, it.probe_keys, it.n_probe,
                                                it.match_positions, it.match_offset, it.match_cnt,
                                                b->fallback_ws[j], b->fallback_ws_bytes[j], ds))
      return st;
  }
  return DTLG_OK;
}

void release(dtlg_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap) cudaStreamDestroy(b->cap);
  cudaFree(b->d_desc);
  cudaFree(b->d_ctl);
  cudaFree(b->d_bucket);
  cudaFree(b->d_mask);
  cudaFree(b->d_items[0]);
  cudaFree(b->d_items[1]);
  for (void* p : b->fallback_ws) cudaFree(p);
}

uint32_t log2_u32(uint32_t v) { return 31u - static_cast<uint32_t>(__builtin_clz(v)); }

// Uploads the descriptor table, every filter staged as planned unless staging is off.
bool upload_desc(dtlg_batch* b) {
  std::vector<BatchDesc> d = b->desc;
  for (size_t f = 0; f < d.size(); f++)
    if (b->staging == 1) d[f].staged = 0;
  return d.empty() ||
         cudaMemcpy(b->d_desc, d.data(), d.size() * sizeof(BatchDesc), cudaMemcpyHostToDevice) == cudaSuccess;
}

}  // namespace

extern "C" {

dtlg_status dtlg_batch_prepare(const dtlg_batch_item* items, uint32_t n_items, int use_graph, dtlg_batch** out) {
  if (!out || (n_items && !items)) return DTLG_ERR_NULL;
  *out = nullptr;
  dtlg_batch* b = new dtlg_batch();
  b->items.assign(items, items + n_items);
  b->use_graph = use_graph != 0;
  std::vector<BatchDesc> desc;
  uint32_t n_probe_tiles = 0, n_ctiles = 0;
  size_t mask_words = 0;
  std::vector<size_t> mask_at;
  for (uint32_t i = 0; i < n_items; i++) {
    const dtlg_batch_item& it = items[i];
    if (!it.filter || !it.filter_words || !it.match_cnt || (it.n_build && !it.build_keys) ||
        (it.n_probe && (!it.probe_keys || !it.match_positions))) {
      delete b;
      return DTLG_ERR_NULL;
    }
    if (it.filter->ck) {  // cuckoo builds synchronize; not part of a batch
      delete b;
      return DTLG_ERR_UNSUPPORTED;
    }
    const int mi = menu_index(it.filter->d);
    const bool aligned = (reinterpret_cast<uintptr_t>(it.build_keys) & 15u) == 0 &&
                         (reinterpret_cast<uintptr_t>(it.probe_keys) & 15u) == 0 &&
                         (reinterpret_cast<uintptr_t>(it.filter_words) & 15u) == 0;
    if (mi < 0 || !aligned) {
      b->fallback.push_back(static_cast<int>(i));
      continue;
    }
    BatchDesc d{};
    d.addr = it.filter->d.addr;
    d.cfg = static_cast<uint32_t>(mi);
    d.words = it.filter_words;
    d.build_keys = it.build_keys;
    d.probe_keys = it.probe_keys;
    d.out = it.match_positions;
    d.count_out = reinterpret_cast<unsigned long long*>(it.match_cnt);
    d.n_build = it.n_build;
    d.n_probe = it.n_probe;
    d.match_offset = it.match_offset;
    d.n_build_tiles = tiles_of(it.n_build);
    d.probe_tile0 = n_probe_tiles;
    d.n_probe_tiles = tiles_of(it.n_probe);
    n_probe_tiles += d.n_probe_tiles;
    d.ctile0 = n_ctiles;
    d.n_ctiles = static_cast<uint32_t>((static_cast<uint64_t>(it.n_probe) + kBatchCompactKeys - 1) / kBatchCompactKeys);
    n_ctiles += d.n_ctiles;
    mask_at.push_back(mask_words);
    mask_words += (static_cast<size_t>(it.n_probe) + 127) / 128 * 4;  // 16-byte aligned per filter
    const uint32_t f = static_cast<uint32_t>(desc.size());
    desc.push_back(d);
  }
  // Staged build: ranges of kBatchRangeBytes; buckets with 25 % + 64 keys of
  // slack over the expected share (overflow takes the direct path).
  size_t bucket_words = 0, cursor_words = 0;
  std::vector<size_t> bucket_at(desc.size()), cursor_at(desc.size());
  for (size_t f = 0; f < desc.size(); f++) {
    BatchDesc& d = desc[f];
    const uint32_t block_bytes = kMenu[d.cfg].wb * kMenu[d.cfg].w;
    const uint32_t bpr = kBatchRangeBytes / block_bytes;  // blocks per range (a power of two)
    const uint32_t n_ranges = (d.addr.block_cnt + bpr - 1) / bpr;
    if (d.n_build == 0 || n_ranges > kBatchMaxRanges) continue;
    d.staged = 1;
    d.n_ranges = n_ranges;
    d.range_shift = log2_u32(bpr);
    d.bucket_cap = static_cast<uint32_t>((static_cast<uint64_t>(d.n_build) * 5 / 4 + n_ranges - 1) / n_ranges) + 64;
    bucket_at[f] = bucket_words;
    cursor_at[f] = cursor_words;
    bucket_words += static_cast<size_t>(n_ranges) * d.bucket_cap;
    cursor_words += n_ranges;
  }
  int dev = 0;
  bool ok = cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occupancy, kBatchedKernel, kBatchThreads,
                                                          kBatchRangeBytes) == cudaSuccess;
  b->occupancy = std::max(1, b->occupancy);
  // The queue: every build tile, then every range item, then every probe
  // tile, each kind in filter order (a filter's probe tiles back to back, so
  // its words stay in L2 while it is probed).  Interleaving the kinds across
  // filters, so that building and probing overlap, measured slower on B200
  // (batched 512-filter step 22.7 vs 20.5 ms): the probes then share L2 with
  // other filters' builds.  Every item depends only on items before it.
  std::vector<uint2> queue[2];
  const uint32_t nf = static_cast<uint32_t>(desc.size());
  for (int v = 0; v < 2; v++) {
    for (uint32_t f = 0; f < nf; f++)
      for (uint32_t t = 0; t < desc[f].n_build_tiles; t++) queue[v].push_back(make_uint2((kItemBuild << 30) | f, t));
    for (uint32_t f = 0; v == 0 && f < nf; f++)
      for (uint32_t r = 0; desc[f].staged && r < desc[f].n_ranges; r++)
        queue[v].push_back(make_uint2((kItemRange << 30) | f, r));
    for (uint32_t f = 0; f < nf; f++)
      for (uint32_t t = 0; t < desc[f].n_probe_tiles; t++)
        queue[v].push_back(make_uint2((kItemProbe << 30) | f, desc[f].probe_tile0 + t));
    for (uint32_t f = 0; f < nf; f++)
      for (uint32_t t = 0; t < desc[f].n_ctiles; t++)
        queue[v].push_back(make_uint2((kItemCompact << 30) | f, desc[f].ctile0 + t));
    b->n_items[v] = static_cast<uint32_t>(queue[v].size());
  }
  b->n_menu = static_cast<uint32_t>(desc.size());
  b->n_probe_tiles = n_probe_tiles;
  b->n_ctiles = n_ctiles;
  b->built_off = 256;
  b->ranges_built_off = b->built_off + round256(static_cast<size_t>(b->n_menu) * 4);
  b->probed_off = b->ranges_built_off + round256(static_cast<size_t>(b->n_menu) * 4);
  b->cursor_off = b->probed_off + round256(static_cast<size_t>(b->n_menu) * 4);
  b->status_off = b->cursor_off + round256(cursor_words * 4);
  b->ctl_bytes = b->status_off + round256(static_cast<size_t>(b->n_ctiles) * 8);
  if (ok && b->n_menu) {
    ok = cudaMalloc(&b->d_ctl, b->ctl_bytes) == cudaSuccess &&
         cudaMalloc(&b->d_bucket, std::max<size_t>(1, bucket_words) * 4) == cudaSuccess &&
         cudaMalloc(&b->d_mask, std::max<size_t>(1, mask_words) * 4) == cudaSuccess &&
         cudaMalloc(&b->d_items[0], std::max<size_t>(1, queue[0].size()) * sizeof(uint2)) == cudaSuccess &&
         cudaMalloc(&b->d_items[1], std::max<size_t>(1, queue[1].size()) * sizeof(uint2)) == cudaSuccess &&
         (queue[0].empty() || cudaMemcpy(b->d_items[0], queue[0].data(), queue[0].size() * sizeof(uint2),
                                         cudaMemcpyHostToDevice) == cudaSuccess) &&
         (queue[1].empty() || cudaMemcpy(b->d_items[1], queue[1].data(), queue[1].size() * sizeof(uint2),
                                         cudaMemcpyHostToDevice) == cudaSuccess);
    for (size_t f = 0; ok && f < desc.size(); f++) desc[f].mask = b->d_mask + mask_at[f];
    for (size_t f = 0; ok && f < desc.size(); f++) {
      if (!desc[f].staged) continue;
      desc[f].bucket = b->d_bucket + bucket_at[f];
      desc[f].cursor = reinterpret_cast<unsigned int*>(b->d_ctl + b->cursor_off) + cursor_at[f];
    }
    b->desc = desc;
  }
  if (ok && b->n_menu) {
    ok = cudaMalloc(&b->d_desc, desc.size() * sizeof(BatchDesc)) == cudaSuccess && upload_desc(b);
  }
  for (size_t j = 0; ok && j < b->fallback.size(); j++) {
    const size_t wsb = dtlg_probe_workspace_size(items[b->fallback[j]].n_probe);
    void* p = nullptr;
    ok = cudaMalloc(&p, wsb) == cudaSuccess;
    b->fallback_ws.push_back(p);
    b->fallback_ws_bytes.push_back(wsb);
  }
  if (!ok) {
    release(b);
    delete b;
    return DTLG_ERR_ALLOC;
  }
  *out = b;
  return DTLG_OK;
}

dtlg_status dtlg_batch_set_ctas_per_sm(dtlg_batch* b, int ctas_per_sm) {
  if (!b) return DTLG_ERR_NULL;
  if (ctas_per_sm < 0) return DTLG_ERR_INVALID_CONFIG;
  b->ctas_per_sm = ctas_per_sm;
  if (b->exec) {  // the grid size is baked into the graph: capture again
    cudaGraphExecDestroy(b->exec);
    cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
  }
  return DTLG_OK;
}

dtlg_status dtlg_batch_run(dtlg_batch* b, dtlg_stream_t stream_) {
  if (!b) return DTLG_ERR_NULL;
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!b->use_graph) return enqueue(b, stream);
  if (!b->warm) {
    // The first run goes straight to the stream: it loads every kernel it
    // touches (module loading is not allowed while a stream is capturing).
    // Later runs replay a graph captured from the second run.
    b->warm = true;
    return enqueue(b, stream);
  }
  if (!b->exec) {
    if (!b->cap && cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess) return DTLG_ERR_CUDA;
    if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return DTLG_ERR_CUDA;
    const dtlg_status st = enqueue(b, b->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &g);
    if (st != DTLG_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return DTLG_ERR_CUDA;
    b->graph = g;
    if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) return DTLG_ERR_CUDA;
  }
  return cudaGraphLaunch(b->exec, stream) == cudaSuccess ? DTLG_OK : DTLG_ERR_CUDA;
}

dtlg_status dtlg_batch_set_staging(dtlg_batch* b, int staging) {
  if (!b) return DTLG_ERR_NULL;
  if (staging < 0 || staging > 1) return DTLG_ERR_INVALID_CONFIG;
  if (staging == b->staging) return DTLG_OK;
  b->staging = staging;
  if (b->n_menu && !upload_desc(b)) return DTLG_ERR_CUDA;
  if (b->exec) {  // the range-queue length is baked into the graph: capture again
    cudaGraphExecDestroy(b->exec);
    cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
  }
  return DTLG_OK;
}

dtlg_status dtlg_batch_autotune(dtlg_batch* b, int reps, dtlg_stream_t stream_, dtlg_batch_plan* best_out) {
  if (!b) return DTLG_ERR_NULL;
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  reps = std::max(1, std::min(reps, 20));
  std::vector<int> ctas = {0};
  for (int c : {2, 3, 4, 6})
    if (c < b->occupancy) ctas.push_back(c);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  dtlg_status st = DTLG_OK;
  dtlg_batch_plan best{b->staging, b->ctas_per_sm, 0.f};
  for (int sg : {0, 1}) {
    for (int c : ctas) {
      if ((st = dtlg_batch_set_staging(b, sg)) || (st = dtlg_batch_set_ctas_per_sm(b, c))) break;
      for (int w = 0; w < 2 && st == DTLG_OK; w++) st = dtlg_batch_run(b, stream_);  // warm + capture
      std::vector<float> ms;
      for (int r = 0; r < reps && st == DTLG_OK; r++) {
        cudaEventRecord(e0, stream);
        st = dtlg_batch_run(b, stream_);
        cudaEventRecord(e1, stream);
        float t = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
          st = DTLG_ERR_CUDA;
        ms.push_back(t);
      }
      if (st != DTLG_OK) break;
      std::sort(ms.begin(), ms.end());
      if (best.ms == 0.f || ms[ms.size() / 2] < best.ms) best = {sg, c, ms[ms.size() / 2]};
    }
    if (st != DTLG_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != DTLG_OK) return st;
  if ((st = dtlg_batch_set_staging(b, best.staging)) || (st = dtlg_batch_set_ctas_per_sm(b, best.ctas_per_sm)))
    return st;
  if (best_out) *best_out = best;
  return DTLG_OK;
}

uint32_t dtlg_batch_staged_count(const dtlg_batch* b) {
  if (!b || b->staging == 1) return 0;
  uint32_t n = 0;
  for (const BatchDesc& d : b->desc) n += d.staged ? 1u : 0u;
  return n;
}

int dtlg_batch_kernel_count(const dtlg_batch* b) {
  if (!b) return 0;
  int n = b->n_menu ? 1 : 0;
  for (int i : b->fallback) {
    const dtlg_batch_item& it = b->items[i];
    n += (it.n_build ? 1 : 0) + dtlg_probe_kernel_count(it.filter, it.n_probe);
  }
  return n;
}

uint32_t dtlg_batch_fallback_count(const dtlg_batch* b) { return b ? static_cast<uint32_t>(b->fallback.size()) : 0; }

void dtlg_batch_destroy(dtlg_batch* b) {
  if (!b) return;
  release(b);
  delete b;
}

}  // extern "C"
