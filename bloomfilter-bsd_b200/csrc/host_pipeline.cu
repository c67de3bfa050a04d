// host_pipeline.cu -- batch_contains / batch_insert over HOST key and position
// buffers, the reference's own calling convention (filter_base.hpp:26,42-45).
//
// Keys are streamed to the device in chunks on a copy stream, probed on the
// caller's stream, and the compacted match positions of each chunk are copied
// back on a second copy stream while later chunks are still in flight:
//   H2D(i+1)  ||  probe(i)  ||  D2H(i-1)
// Chunk i is probed with match_offset + (first key of chunk i), so the
// concatenated outputs are exactly the single-call result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/dtlg.h"

namespace {

constexpr uint64_t kChunk = 1ull << 24;  // keys per chunk (64 MiB)
constexpr int kBufs = 3;

struct Pipeline {
  bool init = false;
  std::mutex mu;
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t keys_in[kBufs], probed[kBufs], out_done[kBufs];
  uint32_t* dkeys[kBufs] = {};
  uint32_t* dpos[kBufs] = {};
  uint64_t* dcnt = nullptr;  // kBufs device counts
  uint64_t* hcnt = nullptr;  // kBufs pinned host counts
  void* ws[kBufs] = {};
  size_t ws_bytes = 0;
};

Pipeline g_pipe[64];
std::mutex g_init_mu;

dtlg_status pipe_for_device(Pipeline** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DTLG_ERR_CUDA;
  Pipeline& p = g_pipe[dev];
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (!p.init) {
    if (cudaStreamCreateWithFlags(&p.h2d, cudaStreamNonBlocking) != cudaSuccess) return DTLG_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&p.d2h, cudaStreamNonBlocking) != cudaSuccess) return DTLG_ERR_CUDA;
    for (int i = 0; i < kBufs; i++) {
      if (cudaEventCreateWithFlags(&p.keys_in[i], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&p.probed[i], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&p.out_done[i], cudaEventDisableTiming) != cudaSuccess)
        return DTLG_ERR_CUDA;
      if (cudaMalloc(&p.dkeys[i], kChunk * 4 + 16) != cudaSuccess) return DTLG_ERR_ALLOC;
      if (cudaMalloc(&p.dpos[i], kChunk * 4 + 16) != cudaSuccess) return DTLG_ERR_ALLOC;
    }
    p.ws_bytes = dtlg_probe_workspace_size(static_cast<uint32_t>(kChunk));
    for (int i = 0; i < kBufs; i++)
      if (cudaMalloc(&p.ws[i], p.ws_bytes) != cudaSuccess) return DTLG_ERR_ALLOC;
    if (cudaMalloc(&p.dcnt, kBufs * sizeof(uint64_t)) != cudaSuccess) return DTLG_ERR_ALLOC;
    if (cudaMallocHost(&p.hcnt, kBufs * sizeof(uint64_t)) != cudaSuccess) return DTLG_ERR_ALLOC;
    p.init = true;
  }
  *out = &p;
  return DTLG_OK;
}

#define PIPE_CUDA(x)                          \
  do {                                        \
    if ((x) != cudaSuccess) return DTLG_ERR_CUDA; \
  } while (0)

}  // namespace

extern "C" {

dtlg_status dtlg_batch_contains_host(const dtlg_filter* f, const uint64_t* words, const uint32_t* keys,
                                     uint64_t n, uint32_t* pos, uint32_t match_offset, uint64_t* match_cnt,
                                     dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!f || !match_cnt || (n && (!keys || !pos))) return DTLG_ERR_NULL;
  *match_cnt = 0;
  if (n == 0) return DTLG_OK;
  Pipeline* p = nullptr;
  if (dtlg_status st = pipe_for_device(&p)) return st;
  std::lock_guard<std::mutex> lk(p->mu);
  // Chunks of kChunk keys, but the last kChunk keys (or fewer) in four
  // pieces: what runs after the last host-to-device copy (its probe and the
  // copy back of its positions) is then a quarter as long.
  const uint64_t full = n > kChunk ? (n - 1) / kChunk : 0;  // whole chunks before the tail
  const uint64_t tail_keys = n - full * kChunk;
  const uint64_t piece = std::max<uint64_t>(1, (tail_keys + 3) / 4);
  const uint64_t chunks = full + (tail_keys + piece - 1) / piece;
  auto chunk_start = [&](uint64_t i) { return i < full ? i * kChunk : full * kChunk + (i - full) * piece; };
  uint64_t written = 0;
  dtlg_status result = DTLG_OK;
  auto drain = [&](uint64_t j) -> dtlg_status {  // copy out the positions of chunk j
    const int b = static_cast<int>(j % kBufs);
    PIPE_CUDA(cudaEventSynchronize(p->probed[b]));
    const uint64_t c = p->hcnt[b];
    if (c == ~0ull) return DTLG_ERR_TIMEOUT;
    PIPE_CUDA(cudaStreamWaitEvent(p->d2h, p->probed[b], 0));
    if (c) PIPE_CUDA(cudaMemcpyAsync(pos + written, p->dpos[b], c * 4, cudaMemcpyDeviceToHost, p->d2h));
    PIPE_CUDA(cudaEventRecord(p->out_done[b], p->d2h));
    written += c;
    return DTLG_OK;
  };
  for (uint64_t i = 0; i < chunks && result == DTLG_OK; i++) {
    const int b = static_cast<int>(i % kBufs);
    const uint64_t start = chunk_start(i);
    const uint32_t len = static_cast<uint32_t>(std::min<uint64_t>(i < full ? kChunk : piece, n - start));
    if (i >= kBufs) {  // buffer b was last used by chunk i - kBufs
      PIPE_CUDA(cudaStreamWaitEvent(p->h2d, p->probed[b], 0));
      PIPE_CUDA(cudaStreamWaitEvent(stream, p->out_done[b], 0));
    }
    PIPE_CUDA(cudaMemcpyAsync(p->dkeys[b], keys + start, static_cast<size_t>(len) * 4, cudaMemcpyHostToDevice,
                              p->h2d));
    PIPE_CUDA(cudaEventRecord(p->keys_in[b], p->h2d));
    PIPE_CUDA(cudaStreamWaitEvent(stream, p->keys_in[b], 0));
    dtlg_status st = dtlg_batch_contains_ws(f, words, p->dkeys[b], len, p->dpos[b],
                                            match_offset + static_cast<uint32_t>(start), p->dcnt + b, p->ws[b],
                                            p->ws_bytes, stream_);
    if (st) return st;
    PIPE_CUDA(cudaMemcpyAsync(p->hcnt + b, p->dcnt + b, 8, cudaMemcpyDeviceToHost, stream));
    PIPE_CUDA(cudaEventRecord(p->probed[b], stream));
    if (i > 0) result = drain(i - 1);
  }
  if (result == DTLG_OK) result = drain(chunks - 1);
  PIPE_CUDA(cudaStreamSynchronize(p->d2h));
  PIPE_CUDA(cudaStreamSynchronize(stream));
  *match_cnt = written;
  return result;
}

dtlg_status dtlg_batch_insert_host(const dtlg_filter* f, uint64_t* words, const uint32_t* keys, uint64_t n,
                                   uint64_t* failed_out, dtlg_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!f || (n && !keys)) return DTLG_ERR_NULL;
  if (failed_out) *failed_out = 0;
  if (n == 0) return DTLG_OK;
  if (dtlg_kind(f) == 2) {
    // cuckoo: one insert over all keys (each call unpacks and repacks the table)
    if (n > 0xFFFFFFFFull) return DTLG_ERR_SIZE;
    uint32_t* d = nullptr;
    PIPE_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d), n * 4 + 16, stream));
    PIPE_CUDA(cudaMemcpyAsync(d, keys, n * 4, cudaMemcpyHostToDevice, stream));
    dtlg_status st = dtlg_batch_insert(f, words, d, static_cast<uint32_t>(n), failed_out, stream_);
    cudaFreeAsync(d, stream);
    PIPE_CUDA(cudaStreamSynchronize(stream));
    return st;
  }
  Pipeline* p = nullptr;
  if (dtlg_status st = pipe_for_device(&p)) return st;
  std::lock_guard<std::mutex> lk(p->mu);
  const uint64_t chunks = (n + kChunk - 1) / kChunk;
  for (uint64_t i = 0; i < chunks; i++) {
    const int b = static_cast<int>(i % kBufs);
    const uint64_t start = i * kChunk;
    const uint32_t len = static_cast<uint32_t>(std::min<uint64_t>(kChunk, n - start));
    if (i >= kBufs) PIPE_CUDA(cudaStreamWaitEvent(p->h2d, p->probed[b], 0));
    PIPE_CUDA(cudaMemcpyAsync(p->dkeys[b], keys + start, static_cast<size_t>(len) * 4, cudaMemcpyHostToDevice,
                              p->h2d));
    PIPE_CUDA(cudaEventRecord(p->keys_in[b], p->h2d));
    PIPE_CUDA(cudaStreamWaitEvent(stream, p->keys_in[b], 0));
    if (dtlg_status st = dtlg_batch_insert(f, words, p->dkeys[b], len, nullptr, stream_)) return st;
    PIPE_CUDA(cudaEventRecord(p->probed[b], stream));
  }
  PIPE_CUDA(cudaStreamSynchronize(stream));
  return DTLG_OK;
}

}  // extern "C"
