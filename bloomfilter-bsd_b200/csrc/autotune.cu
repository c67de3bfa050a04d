// autotune.cu -- picks a filter's probe plan by timing the alternatives on
// the GPU, with the caller's filter and keys.
//
// The reference tunes its SIMD kernels the same way: every unroll factor is
// timed on random keys and the fastest is kept per configuration
// (blocked_bloomfilter_tune_impl.hpp:162-268, cuckoofilter_tune_impl.hpp:
// 118-225).  Here the alternatives are the probe plans -- the fused kernel,
// the bitmask kernel in one or more block-range passes with either register
// budget, (Bloom and blocked cuckoo filters beyond 32 MiB) the partitioned
// probe, and (Bloom filters of at most 192 KiB) the shared-memory probe -- and the
// choice is stored on the filter handle.  Every plan must report the same
// match count; a disagreement is returned as an error.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/dtlg.h"
#include "filter_handle.hpp"

namespace {

struct Plan {
  int mode, variant, passes;
};

std::vector<Plan> candidate_plans(const dtlg_filter* f, uint32_t n) {
  const uint64_t bytes = (f->d.m_actual + 7) / 8;
  std::vector<Plan> out;
  out.push_back({1, -1, 0});
  if (n >= 4096) {
    std::vector<int> passes = {1};
    if (bytes > (64ull << 20)) passes.insert(passes.end(), {2, 4});
    if (bytes > (512ull << 20)) passes.push_back(8);
    for (int v = 0; v < dtlg::kBitsVariants; v++)
      for (int p : passes) out.push_back({2, v, p});
    if (f->pk->probe_smem && bytes <= (192ull << 10)) out.push_back({4, -1, 0});
    if (f->pk->probe_pairs[0] && bytes > (32ull << 20))
      for (int v = 0; v < dtlg::kBitsVariants; v++) out.push_back({3, v, 0});
  }
  return out;
}

}  // namespace

extern "C" {

dtlg_status dtlg_autotune_probe(dtlg_filter* f, const uint64_t* filter_words, const uint32_t* keys, uint32_t n,
                                uint32_t* match_positions, int reps, dtlg_stream_t stream_,
                                dtlg_probe_plan* best_out) {
  if (!f || !filter_words || !keys || !match_positions) return DTLG_ERR_NULL;
  if (n == 0) return DTLG_ERR_INVALID_CONFIG;
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  reps = std::max(1, std::min(reps, 50));
  const size_t ws_bytes = dtlg_probe_workspace_size(n);
  void* ws = nullptr;
  uint64_t* cnt = nullptr;
  DTLG_TRY_CUDA(cudaMalloc(&ws, ws_bytes));
  if (cudaMalloc(&cnt, sizeof(uint64_t)) != cudaSuccess) {
    cudaFree(ws);
    return DTLG_ERR_ALLOC;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int saved_mode = f->probe_mode, saved_variant = f->bits_variant, saved_passes = f->probe_passes;
  dtlg_status st = DTLG_OK;
  dtlg_probe_plan best{0, -1, 0, 0.f, 0.f};
  uint64_t want = ~0ull;
  for (const Plan& p : candidate_plans(f, n)) {
    f->probe_mode = p.mode;
    f->bits_variant = p.variant;
    f->probe_passes = p.passes;
    st = dtlg_batch_contains_ws(f, filter_words, keys, n, match_positions, 0, cnt, ws, ws_bytes, stream_);
    uint64_t got = 0;
    if (st == DTLG_OK && cudaMemcpyAsync(&got, cnt, 8, cudaMemcpyDeviceToHost, stream) != cudaSuccess)
      st = DTLG_ERR_CUDA;
    if (st == DTLG_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = DTLG_ERR_CUDA;
    if (st != DTLG_OK) break;
    if (got == ~0ull) {
      st = DTLG_ERR_TIMEOUT;
      break;
    }
    if (want == ~0ull) want = got;
    if (got != want) {  // all plans compute the same result
      st = DTLG_ERR_CUDA;
      break;
    }
    std::vector<float> ms;
    for (int r = 0; r < reps && st == DTLG_OK; r++) {
      cudaEventRecord(e0, stream);
      st = dtlg_batch_contains_ws(f, filter_words, keys, n, match_positions, 0, cnt, ws, ws_bytes, stream_);
      cudaEventRecord(e1, stream);
      float t = 0.f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
        st = DTLG_ERR_CUDA;
      ms.push_back(t);
    }
    if (st != DTLG_OK) break;
    std::sort(ms.begin(), ms.end());
    const float med = ms[ms.size() / 2];
    if (best.ms == 0.f || med < best.ms) best = {p.mode, p.variant, p.passes, med, 0.f};
  }
  if (st == DTLG_OK) {
    f->probe_mode = best.mode;
    f->bits_variant = best.variant;
    f->probe_passes = best.passes;
    best.gkeys_per_s = best.ms > 0.f ? static_cast<float>(n) / (best.ms * 1e6f) : 0.f;
    if (best_out) *best_out = best;
  } else {
    f->probe_mode = saved_mode;
    f->bits_variant = saved_variant;
    f->probe_passes = saved_passes;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(ws);
  cudaFree(cnt);
  return st;
}

}  // extern "C"
