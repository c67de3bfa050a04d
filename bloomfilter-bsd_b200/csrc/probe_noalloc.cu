// probe_noalloc.cu -- batch_contains for callers that cannot allocate device memory.
//
// Some callers of a probe cannot call cudaMalloc: a query engine whose device
// memory is all handed out up front by its own buffer manager, a plugin living
// inside a host application that owns the GPU's memory, or a latency-critical
// path where a cudaMalloc (which may synchronize the device and take
// milliseconds) is not acceptable.  They still bring their own inputs and
// outputs; what they cannot provide is the probe's scratch memory (the tile
// queue and the per-tile look-back words of the ordered compaction).
//
// dtlg_batch_contains_noalloc keeps that scratch in one file-scope device
// array, kNoAllocScratchBytes (~128 KiB) per GPU, which every GPU that loads
// the library holds until the process exits.  It serves at most
// DTLG_NOALLOC_MAX_KEYS keys per call.  All calls on a device share the array
// and it keeps the last call's contents, so each call first clears the part it
// uses; two calls whose kernels overlap on the GPU (different streams without
// ordering between them, or several host threads) race on it and must be
// serialized by the caller.
//
// It always runs the fused single-kernel probe (plan 1): the scratch has no
// room for the match bitmask or the key pairs of the other plans, so filters
// far beyond L2 probe slower here than through dtlg_batch_contains_async, with
// the same results.  A look-back wait that gives up leaves UINT64_MAX in
// *match_cnt_dev (the error word itself stays in the shared scratch).  The
// array's device address is resolved once per device and kept for the life of
// the process; after a cudaDeviceReset it would be stale, so the entry point
// is not for processes that reset their devices.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/dtlg.h"
#include "filter_handle.hpp"
#include "registry.hpp"

namespace {

using namespace dtlg;

// scratch layout: 128-byte header (tile counter, error word), then one 64-bit
// look-back word per tile of the largest call
struct NoAllocHeader {
  unsigned int tile_ctr;
  unsigned int err;
  unsigned long long pad[15];
};
static_assert(sizeof(NoAllocHeader) == 128, "one 128-byte line");

constexpr uint64_t kMaxTiles = (static_cast<uint64_t>(DTLG_NOALLOC_MAX_KEYS) + 3 + kProbeTile - 1) / kProbeTile;
constexpr uint64_t kNoAllocScratchBytes = ((sizeof(NoAllocHeader) + kMaxTiles * 8 + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_probe_scratch[kNoAllocScratchBytes];

struct DeviceScratch {
  bool ready = false;
  void* ptr = nullptr;  // device address of g_probe_scratch on this device
  int sms = 0;
};
std::mutex g_mu;
DeviceScratch g_scratch[64];

// Once per device, with that device current: the host-side name of a
// __device__ array is only a stand-in, so the kernel gets the address that
// cudaGetSymbolAddress reports for this device.
dtlg_status scratch_for_current_device(DeviceScratch** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DTLG_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceScratch& s = g_scratch[dev];
  if (!s.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_probe_scratch) != cudaSuccess || p == nullptr) return DTLG_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return DTLG_ERR_CUDA;
    s.ptr = p;
    s.sms = sms;
    s.ready = true;
  }
  *out = &s;
  return DTLG_OK;
}

}  // namespace

extern "C" dtlg_status dtlg_batch_contains_noalloc(const dtlg_filter* f, const uint64_t* filter_words,
                                                   const uint32_t* keys, uint32_t key_cnt,
                                                   uint32_t* match_positions, uint32_t match_offset,
                                                   uint64_t* match_cnt_dev, dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!f || !filter_words || !match_cnt_dev || (key_cnt && (!keys || !match_positions))) return DTLG_ERR_NULL;
  if (reinterpret_cast<uintptr_t>(filter_words) & 15u) return DTLG_ERR_ALIGNMENT;
  if (key_cnt > DTLG_NOALLOC_MAX_KEYS) return DTLG_ERR_WORKSPACE;
  DeviceScratch* s = nullptr;
  if (dtlg_status st = scratch_for_current_device(&s)) return st;
  if (key_cnt == 0) {
    return cudaMemsetAsync(match_cnt_dev, 0, sizeof(uint64_t), stream) == cudaSuccess ? DTLG_OK : DTLG_ERR_CUDA;
  }
  const uint32_t pre = static_cast<uint32_t>((reinterpret_cast<uintptr_t>(keys) & 15u) >> 2);
  const uint64_t n_phys = static_cast<uint64_t>(key_cnt) + pre;
  const uint32_t tiles = static_cast<uint32_t>((n_phys + kProbeTile - 1) / kProbeTile);
  const size_t used = sizeof(NoAllocHeader) + static_cast<size_t>(tiles) * 8;
  // the array keeps the previous call's words: clear the counter, the error
  // word and the status words this call will read
  if (cudaMemsetAsync(s->ptr, 0, used, stream) != cudaSuccess) return DTLG_ERR_CUDA;
  NoAllocHeader* h = static_cast<NoAllocHeader*>(s->ptr);
  ProbeArgs a{};
  a.filter = filter_words;
  a.keys_al = keys - pre;
  a.n_phys = n_phys;
  a.pre = pre;
  a.match_offset = match_offset;
  a.out = match_positions;
  a.count_out = reinterpret_cast<unsigned long long*>(match_cnt_dev);
  a.status = reinterpret_cast<unsigned long long*>(h + 1);
  a.tile_ctr = &h->tile_ctr;
  a.err = &h->err;
  a.n_tiles = tiles;
  set_filter_args(f->d, &a);
  // 256-bit block loads where the words are 32-byte aligned (as every plan of
  // dtlg_batch_contains_async reads them)
  a.vec32 = (reinterpret_cast<uintptr_t>(filter_words) & 31u) == 0 ? 1u : 0u;
  const probe_fn fn = f->pk->probe;
  const occ_fn occ = f->pk->probe_blocks_per_sm;
  const int per_sm = std::max(1, occ());
  const int grid = static_cast<int>(std::min<uint64_t>(tiles, static_cast<uint64_t>(s->sms) * per_sm));
  return fn(a, grid, stream) == cudaSuccess ? DTLG_OK : DTLG_ERR_CUDA;
}
