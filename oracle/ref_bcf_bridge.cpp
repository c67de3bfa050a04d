// ref_bcf_bridge.cpp -- C entry points over the reference's blocked cuckoo
// filter, dtl::bcf (src/dtl/filter/bcf.hpp:11-63, bcf.cpp:9-93).
//
// TEST INFRASTRUCTURE ONLY.  No reference code lives here: oracle/Makefile
// compiles the reference's own bcf.cpp from its place in the reference tree
// together with this file.  Two builds: libdtlref_bcf.so for a plain x86-64
// target (every config takes the scalar batch path of
// blocked_cuckoofilter_logic.hpp:120-170) and libdtlref_bcf_avx2.so, where
// the <16,4> and <8,4> configs take the AVX2 batch path of
// blocked_cuckoofilter_simd.hpp instead.
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "dtl/filter/bcf.hpp"

extern "C" {

void* ref_bcf_create(uint64_t m, uint32_t block_bytes, uint32_t tag_bits, uint32_t assoc) {
  try {
    return new dtl::bcf(m, block_bytes, tag_bits, assoc);
  } catch (...) {
    return nullptr;
  }
}

void ref_bcf_destroy(void* h) { delete static_cast<dtl::bcf*>(h); }

uint64_t ref_bcf_size(void* h) { return static_cast<dtl::bcf*>(h)->size(); }
uint64_t ref_bcf_size_in_bytes(void* h) { return static_cast<dtl::bcf*>(h)->size_in_bytes(); }

size_t ref_bcf_name(void* h, char* buf, size_t cap) {
  const std::string s = static_cast<dtl::bcf*>(h)->name();
  if (buf && cap > s.size()) std::memcpy(buf, s.c_str(), s.size() + 1);
  return s.size();
}

int ref_bcf_batch_insert(void* h, uint32_t* data, const uint32_t* keys, uint32_t n) {
  return static_cast<dtl::bcf*>(h)->batch_insert(data, keys, n) ? 1 : 0;
}

int ref_bcf_contains(void* h, const uint32_t* data, uint32_t key) {
  return static_cast<dtl::bcf*>(h)->contains(data, key) ? 1 : 0;
}

uint64_t ref_bcf_batch_contains(void* h, const uint32_t* data, const uint32_t* keys, uint32_t n,
                                uint32_t* out, uint32_t off) {
  return static_cast<dtl::bcf*>(h)->batch_contains(data, keys, n, out, off);
}

// Multi-threaded probe in the shape of model/benchmark.cpp:123-165: each
// thread probes its own contiguous slice in batches of 1024 keys
// (batchwise.hpp:9) into its own slice of the output buffer.
uint64_t ref_bcf_batch_contains_mt(void* h, const uint32_t* data, const uint32_t* keys, uint64_t n,
                                   uint32_t* out, int threads) {
  dtl::bcf* f = static_cast<dtl::bcf*>(h);
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
        c += f->batch_contains(data, keys + i, len, out + b + c, (uint32_t)i);
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
uint64_t ref_bcf_batch_contains_mt_list(void* h, const uint32_t* data, const uint32_t* keys, uint64_t n,
                                   uint32_t* out, int threads) {
  dtl::bcf* f = static_cast<dtl::bcf*>(h);
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
        c += f->batch_contains(data, keys + i, len, out + b + c, (uint32_t)i);
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
