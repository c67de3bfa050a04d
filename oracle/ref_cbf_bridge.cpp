// ref_cbf_bridge.cpp -- C entry points over the reference's classic Bloom
// filter, dtl::bloomfilter_logic<uint32_t, addressing>
// (src/dtl/filter/bloomfilter/bloomfilter_logic.hpp:22-212).
//
// TEST INFRASTRUCTURE ONLY.  No reference code lives here: the reference's
// header is included from its place in the reference tree (oracle/Makefile
// sets the include path) and instantiated for both addressing modes, as a
// user of that header-only template does.  Its batch_contains is scalar.
#include <cstring>
#include <cstdint>
#include <thread>
#include <vector>

#include <dtl/dtl.hpp>
#include <dtl/simd.hpp>
#include <dtl/simd/extensions.hpp>
#include <dtl/filter/bloomfilter/bloomfilter_logic.hpp>

namespace {
using pow2_t = dtl::bloomfilter_logic<uint32_t, dtl::block_addressing::POWER_OF_TWO>;
using magic_t = dtl::bloomfilter_logic<uint32_t, dtl::block_addressing::MAGIC>;
struct handle {
  pow2_t* p = nullptr;
  magic_t* g = nullptr;
};
}  // namespace

extern "C" {

void* ref_cbf_create(uint64_t m, uint32_t k, uint32_t magic) {
  try {
    handle* h = new handle();
    if (magic) h->g = new magic_t(m, k);
    else h->p = new pow2_t(m, k);
    return h;
  } catch (...) {
    return nullptr;
  }
}

void ref_cbf_destroy(void* v) {
  handle* h = static_cast<handle*>(v);
  delete h->p;
  delete h->g;
  delete h;
}

uint64_t ref_cbf_size(void* v) {
  handle* h = static_cast<handle*>(v);
  return h->p ? h->p->size() : h->g->size();
}

uint64_t ref_cbf_length(void* v) {
  handle* h = static_cast<handle*>(v);
  return h->p ? h->p->get_length() : h->g->get_length();
}

// Returns 0 when the reference throws (hash_no > 16).
int ref_cbf_batch_insert(void* v, uint32_t* data, const uint32_t* keys, uint32_t n) {
  handle* h = static_cast<handle*>(v);
  try {
    if (h->p) h->p->batch_insert(data, keys, n);
    else h->g->batch_insert(data, keys, n);
    return 1;
  } catch (...) {
    return 0;
  }
}

uint64_t ref_cbf_batch_contains(void* v, const uint32_t* data, const uint32_t* keys, uint32_t n, uint32_t* out,
                                uint32_t off) {
  handle* h = static_cast<handle*>(v);
  return h->p ? h->p->batch_contains(data, keys, n, out, off) : h->g->batch_contains(data, keys, n, out, off);
}

// Multi-threaded probe in the shape of model/benchmark.cpp:123-165.
uint64_t ref_cbf_batch_contains_mt(void* v, const uint32_t* data, const uint32_t* keys, uint64_t n,
                                   uint32_t* out, int threads) {
  if (threads < 1) threads = 1;
  std::vector<uint64_t> cnt(threads, 0);
  std::vector<std::thread> th;
  for (int t = 0; t < threads; t++) {
    th.emplace_back([=, &cnt]() {
      const uint64_t b = n * (uint64_t)t / (uint64_t)threads;
      const uint64_t e = n * (uint64_t)(t + 1) / (uint64_t)threads;
      uint64_t c = 0;
      for (uint64_t i = b; i < e; i += 1024) {
        const uint32_t len = (uint32_t)std::min<uint64_t>(1024, e - i);
        c += ref_cbf_batch_contains(v, data, keys + i, len, out + b + c, (uint32_t)i);
      }
      cnt[t] = c;
    });
  }
  uint64_t total = 0;
  for (int t = 0; t < threads; t++) {
    th[t].join();
    total += cnt[t];
  }
  return total;
}

// As above, then the slices' lists moved together into the one ascending
// list (positions i) that a single batch_contains over all n keys returns.
uint64_t ref_cbf_batch_contains_mt_list(void* v, const uint32_t* data, const uint32_t* keys, uint64_t n,
                                   uint32_t* out, int threads) {
  if (threads < 1) threads = 1;
  std::vector<uint64_t> cnt(threads, 0);
  std::vector<std::thread> th;
  for (int t = 0; t < threads; t++) {
    th.emplace_back([=, &cnt]() {
      const uint64_t b = n * (uint64_t)t / (uint64_t)threads;
      const uint64_t e = n * (uint64_t)(t + 1) / (uint64_t)threads;
      uint64_t c = 0;
      for (uint64_t i = b; i < e; i += 1024) {
        const uint32_t len = (uint32_t)std::min<uint64_t>(1024, e - i);
        c += ref_cbf_batch_contains(v, data, keys + i, len, out + b + c, (uint32_t)i);
      }
      cnt[t] = c;
    });
  }
  for (auto& x : th) x.join();
  uint64_t total = 0;
  for (int t = 0; t < threads; t++) {
    const uint64_t b = n * (uint64_t)t / (uint64_t)threads;
    if (total != b && cnt[t]) std::memmove(out + total, out + b, cnt[t] * sizeof(uint32_t));
    total += cnt[t];
  }
  return total;
}

}  // extern "C"
