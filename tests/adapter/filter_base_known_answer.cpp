// Drives the GPU adapter (bloomfilter-bsd_b200/adapter/gpu_filter.hpp) through
// the reference's own interface, dtl::filter::filter_base, by virtual calls
// only, and checks the reference's known answer (src/dtl/filter/filter_test.cpp:
// 16-40): keys {13, 37, 42, 88} inserted into the default blocked Bloom filter
// config at m = 1024 are found at positions [0, 1, 2, 3]; probing
// {0, 1, 42, 2} with match offset 1000 gives [1002].  Then the same calls for
// a sectorized, a zoned and a cuckoo filter (every member found, ascending
// positions), the single-key members, size(), name(), and the exception the
// reference throws for an invalid config.  Prints "OK" and exits 0 on success.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <vector>

#include "gpu_filter.hpp"

using dtl::filter::filter_base;
using dtlg::adapter::gpu_filter;
using dtlg::adapter::gpu_filter_data;

#define CHECK(c)                                                  \
  do {                                                            \
    if (!(c)) {                                                   \
      std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #c); \
      std::exit(1);                                               \
    }                                                             \
  } while (0)

template <class T>
struct dev_vec {
  T* p = nullptr;
  explicit dev_vec(const std::vector<T>& h) {
    CHECK(cudaMalloc(reinterpret_cast<void**>(&p), (h.size() + 1) * sizeof(T)) == cudaSuccess);
    CHECK(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess);
  }
  explicit dev_vec(std::size_t n) { CHECK(cudaMalloc(reinterpret_cast<void**>(&p), (n + 1) * sizeof(T)) == cudaSuccess); }
  ~dev_vec() { cudaFree(p); }
  std::vector<T> get(std::size_t n) const {
    std::vector<T> h(n);
    CHECK(cudaMemcpy(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess);
    return h;
  }
};

// The reference's known answer, through a filter_base*.
static void known_answer(filter_base& f, filter_base::word_t* data) {
  dev_vec<uint32_t> keys(std::vector<uint32_t>{13, 37, 42, 88});
  CHECK(f.batch_insert(data, keys.p, 4));
  dev_vec<uint32_t> pos(4);
  CHECK(f.batch_contains(data, keys.p, 4, pos.p, 0) == 4);
  CHECK((pos.get(4) == std::vector<uint32_t>{0, 1, 2, 3}));
  dev_vec<uint32_t> probe(std::vector<uint32_t>{0, 1, 42, 2});
  CHECK(f.batch_contains(data, probe.p, 4, pos.p, 1000) == 1);
  CHECK(pos.get(1)[0] == 1002);
  CHECK(f.contains(data, 42) && !f.contains(data, 0));
}

// Every member found at its ascending position, for a larger build.
static void members(filter_base& f, filter_base::word_t* data, uint32_t n) {
  std::vector<uint32_t> h(n);
  for (uint32_t i = 0; i < n; i++) h[i] = i * 2654435761u + 12345u;
  dev_vec<uint32_t> keys(h);
  CHECK(f.batch_insert(data, keys.p, n));
  dev_vec<uint32_t> pos(n);
  CHECK(f.batch_contains(data, keys.p, n, pos.p, 7) == n);
  const std::vector<uint32_t> got = pos.get(n);
  for (uint32_t i = 0; i < n; i++) CHECK(got[i] == i + 7);
  CHECK(f.insert(data, 99991u) && f.contains(data, 99991u));
}

int main() {
  {  // filter_test.cpp:18-21: the default blocked_bloomfilter_config, m = 1024
    dtlg_bloom_config c{8, 4, 1, 1, 0, 1};
    std::unique_ptr<filter_base> f(new gpu_filter(c, 1024));
    gpu_filter_data d(static_cast<const gpu_filter&>(*f));
    CHECK(f->size() == d.words() && f->size_in_bytes() == 128);
    CHECK(f->name().find("\"name\":\"blocked_bloom_multiword\"") != std::string::npos);
    known_answer(*f, d.data());
  }
  {  // sectorized u64 w=8 s=8 k=8 (MAGIC addressing), zoned u32 w=16 z=4 k=8
    dtlg_bloom_config s8{8, 8, 8, 8, 0, 1}, z4{8, 4, 16, 16, 0, 4};
    for (const dtlg_bloom_config& c : {s8, z4}) {
      std::unique_ptr<filter_base> f(new gpu_filter(c, 12 * 50000 + 3));
      gpu_filter_data d(static_cast<const gpu_filter&>(*f));
      members(*f, d.data(), 50000);
    }
  }
  {  // cuckoo t=16 b=4
    dtlg_cuckoo_config c{16, 4, 0};
    std::unique_ptr<filter_base> f(new gpu_filter(c, 1 << 20));
    gpu_filter_data d(static_cast<const gpu_filter&>(*f));
    members(*f, d.data(), 40000);
  }
  {  // an invalid config throws std::invalid_argument, as the reference's constructor
    bool threw = false;
    try {
      dtlg_bloom_config bad{3, 4, 2, 2, 0, 1};  // k = 3 is not a multiple of s = 2
      gpu_filter g(bad, 1024);
    } catch (const std::invalid_argument&) {
      threw = true;
    }
    CHECK(threw);
  }
  std::printf("OK\n");
  return 0;
}
