// ref_bridge.cpp -- registry and C ABI of the reference oracle library.
// TEST INFRASTRUCTURE ONLY (see ref_bridge.hpp).
#include "ref_bridge.hpp"

#include <algorithm>
#include <mutex>

namespace refbridge {

static std::vector<entry>& blooms() { static std::vector<entry> v; return v; }
static std::vector<entry>& cuckoos() { static std::vector<entry> v; return v; }
void register_bloom(const entry& e) { blooms().push_back(e); }
void register_cuckoo(const entry& e) { cuckoos().push_back(e); }

struct handle {
  const ops* o;
  void* logic;
};

}  // namespace refbridge

using namespace refbridge;

extern "C" {

int ref_simd_lanes() { return (int)kLanes; }

// dtl::next_cheap_magic (div.hpp:30-57); returns 0 when it throws.
int ref_next_cheap_magic(uint32_t n, uint32_t* divisor, uint32_t* magic, uint32_t* shift) {
  try {
    dtl::fast_divisor_u32_t d = dtl::next_cheap_magic(n);
    *divisor = d.divisor;
    *magic = d.magic;
    *shift = d.shift_amount;
    return 1;
  } catch (...) {
    return 0;
  }
}

// Addressing follows the dispatchers: POW2 iff m is a power of two
// (blocked_bloomfilter.hpp:234-242, cuckoofilter.hpp:211-213).
static uint32_t addr_of(uint64_t m) { return dtl::is_power_of_two(m) ? 0u : 1u; }

void* ref_bloom_create(uint32_t word_bytes, uint32_t w, uint32_t s, uint32_t z, uint32_t k,
                       uint64_t m) {
  const uint32_t a = addr_of(m);
  for (const entry& e : blooms()) {
    if (e.a == word_bytes && e.b == w && e.c == s && e.d == z && e.e == k && e.addr == a) {
      try {
        void* l = e.o->create(m);
        return new handle{e.o, l};
      } catch (...) {
        return nullptr;
      }
    }
  }
  return nullptr;
}

void* ref_cuckoo_create(uint32_t t, uint32_t b, uint64_t m) {
  const uint32_t a = addr_of(m);
  for (const entry& e : cuckoos()) {
    if (e.a == t && e.b == b && e.addr == a) {
      try {
        void* l = e.o->create(m);
        return new handle{e.o, l};
      } catch (...) {
        return nullptr;
      }
    }
  }
  return nullptr;
}

int ref_instance_count(int cuckoo) { return (int)(cuckoo ? cuckoos().size() : blooms().size()); }

void ref_destroy(void* h) {
  if (!h) return;
  handle* x = static_cast<handle*>(h);
  x->o->destroy(x->logic);
  delete x;
}

uint64_t ref_word_cnt(void* h) { handle* x = static_cast<handle*>(h); return x->o->word_cnt(x->logic); }
uint64_t ref_length(void* h) { handle* x = static_cast<handle*>(h); return x->o->length(x->logic); }

int ref_insert(void* h, void* data, const uint32_t* keys, uint32_t n) {
  handle* x = static_cast<handle*>(h);
  return x->o->insert(x->logic, data, keys, n);
}

int ref_contains(void* h, const void* data, uint32_t key) {
  handle* x = static_cast<handle*>(h);
  return x->o->contains(x->logic, data, key);
}

uint64_t ref_batch_contains(void* h, const void* data, const uint32_t* keys, uint32_t n,
                            uint32_t* out, uint32_t off, int unroll) {
  handle* x = static_cast<handle*>(h);
  return x->o->batch_contains(x->logic, data, keys, n, out, off, unroll);
}

uint64_t ref_count_occupied(void* h, const void* data) {
  handle* x = static_cast<handle*>(h);
  return x->o->count_occupied(x->logic, data);
}

// Multi-threaded probe in the shape of model/benchmark.cpp:123-165: each
// thread probes its own contiguous slice in batches of 1024 keys
// (batchwise.hpp:9) into its own slice of the output buffer.  Returns the
// total match count.
uint64_t ref_batch_contains_mt(void* h, const void* data, const uint32_t* keys, uint64_t n,
                               uint32_t* out, int threads, int unroll) {
  handle* x = static_cast<handle*>(h);
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
        c += x->o->batch_contains(x->logic, data, keys + i, len, out + b + c, (uint32_t)i, unroll);
      }
      cnt[t] = c;
    });
  }
  uint64_t total = 0;
  for (int t = 0; t < threads; t++) { th[t].join(); total += cnt[t]; }
  return total;
}

// As ref_batch_contains_mt, then the threads' lists moved together: thread t
// probed slice [b_t, e_t) and wrote its c_t positions at out + b_t, so moving
// the slices down in thread order gives the one ascending list a single
// batch_contains over all n keys returns (positions i, no offset).
uint64_t ref_batch_contains_mt_list(void* h, const void* data, const uint32_t* keys, uint64_t n,
                                    uint32_t* out, int threads, int unroll) {
  handle* x = static_cast<handle*>(h);
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
        c += x->o->batch_contains(x->logic, data, keys + i, len, out + b + c, (uint32_t)i, unroll);
      }
      cnt[t] = c;
    });
  }
  for (auto& t : th) t.join();
  uint64_t total = 0;
  for (int t = 0; t < threads; t++) {
    const uint64_t b = n * (uint64_t)t / (uint64_t)threads;
    if (total != b && cnt[t]) std::memmove(out + total, out + b, cnt[t] * sizeof(uint32_t));
    total += cnt[t];
  }
  return total;
}

// Multi-threaded Bloom build: the sgew/sltw inserts are CAS-based and may run
// concurrently (blocked_bloomfilter_block_logic_sgew.hpp:300-325).
void ref_insert_mt(void* h, void* data, const uint32_t* keys, uint64_t n, int threads) {
  handle* x = static_cast<handle*>(h);
  if (threads < 1) threads = 1;
  std::vector<std::thread> th;
  for (int t = 0; t < threads; t++) {
    th.emplace_back([=]() {
      const uint64_t b = n * (uint64_t)t / (uint64_t)threads;
      const uint64_t e = n * (uint64_t)(t + 1) / (uint64_t)threads;
      for (uint64_t i = b; i < e; i += (1u << 20)) {
        const uint32_t len = (uint32_t)std::min<uint64_t>(1u << 20, e - i);
        x->o->insert(x->logic, data, keys + i, len);
      }
    });
  }
  for (auto& t : th) t.join();
}

}  // extern "C"
