// gpu_filter.cpp -- dtl::filter::filter_base over libdtlg.so (see gpu_filter.hpp).
#include "gpu_filter.hpp"

#include <cstdio>
#include <exception>
#include <utility>
#include <vector>

namespace dtlg {
namespace adapter {

void throw_status(dtlg_status st, const char* what) {
  switch (st) {
    case DTLG_OK:
      return;
    case DTLG_ERR_INVALID_CONFIG:  // the reference's constructors: std::invalid_argument
      throw std::invalid_argument(std::string(what) + ": " + dtlg_status_string(st));
    case DTLG_ERR_SIZE:            // "block count must not exceed 2^32": std::logic_error
      throw std::logic_error(std::string(what) + ": " + dtlg_status_string(st));
    default:
      throw std::runtime_error(std::string(what) + ": " + dtlg_status_string(st));
  }
}

gpu_filter::gpu_filter(const dtlg_bloom_config& config, std::size_t m, cudaStream_t stream) : stream_(stream) {
  throw_status(dtlg_bloom_create(&config, m, &f_), "dtlg_bloom_create");
}

gpu_filter::gpu_filter(const dtlg_cuckoo_config& config, std::size_t m, cudaStream_t stream) : stream_(stream) {
  throw_status(dtlg_cuckoo_create(&config, m, &f_), "dtlg_cuckoo_create");
}

gpu_filter::~gpu_filter() { dtlg_destroy(f_); }

gpu_filter::gpu_filter(gpu_filter&& o) noexcept : f_(o.f_), stream_(o.stream_) { o.f_ = nullptr; }

gpu_filter& gpu_filter::operator=(gpu_filter&& o) noexcept {
  std::swap(f_, o.f_);
  std::swap(stream_, o.stream_);
  return *this;
}

dtl::filter::filter_base& gpu_filter::operator=(dtl::filter::filter_base&& o) noexcept {
  gpu_filter* g = dynamic_cast<gpu_filter*>(&o);
  if (!g) {
    // a CPU filter's state cannot become a GPU filter's; the base declares
    // this assignment noexcept, so misuse ends the program
    std::fprintf(stderr, "gpu_filter: move-assignment from another filter type\n");
    std::terminate();
  }
  return *this = std::move(*g);
}

$u1 gpu_filter::insert(word_t* __restrict filter_data, key_t key) {
  throw_status(dtlg_insert(f_, filter_data, key, reinterpret_cast<dtlg_stream_t>(stream_)), "dtlg_insert");
  return true;
}

// Bloom inserts always succeed (bbf_32.cpp:38-46); a cuckoo insert that could
// not place a key returns false (cuckoofilter_logic.hpp:330-337).
$u1 gpu_filter::batch_insert(word_t* __restrict filter_data, const key_t* __restrict keys, u32 key_cnt) {
  const dtlg_status st =
      dtlg_batch_insert(f_, filter_data, keys, key_cnt, nullptr, reinterpret_cast<dtlg_stream_t>(stream_));
  if (st == DTLG_ERR_CUCKOO_FULL) return false;
  throw_status(st, "dtlg_batch_insert");
  return true;
}

$u1 gpu_filter::contains(const word_t* __restrict filter_data, key_t key) const {
  int r = 0;
  throw_status(dtlg_contains(f_, filter_data, key, &r, reinterpret_cast<dtlg_stream_t>(stream_)), "dtlg_contains");
  return r != 0;
}

$u64 gpu_filter::batch_contains(const word_t* __restrict filter_data, const key_t* __restrict keys, u32 key_cnt,
                                $u32* __restrict match_positions, u32 match_offset) const {
  uint64_t cnt = 0;
  throw_status(dtlg_batch_contains(f_, filter_data, keys, key_cnt, match_positions, match_offset, &cnt,
                                   reinterpret_cast<dtlg_stream_t>(stream_)),
               "dtlg_batch_contains");
  return cnt;
}

std::string gpu_filter::name() const {
  std::vector<char> buf(256);
  std::size_t n = dtlg_name(f_, buf.data(), buf.size());
  if (n >= buf.size()) {
    buf.resize(n + 1);
    n = dtlg_name(f_, buf.data(), buf.size());
  }
  return std::string(buf.data(), n);
}

std::size_t gpu_filter::size_in_bytes() const { return dtlg_size_in_bytes(f_); }
std::size_t gpu_filter::size() const { return dtlg_size(f_); }
std::size_t gpu_filter::alloc_words() const { return dtlg_alloc_words_u64(f_); }

gpu_filter_data::gpu_filter_data(const gpu_filter& f) : n_(f.alloc_words()) {
  if (cudaMalloc(reinterpret_cast<void**>(&words_), n_ * sizeof(*words_)) != cudaSuccess)
    throw std::runtime_error("gpu_filter_data: cudaMalloc failed");
  if (cudaMemset(words_, 0, n_ * sizeof(*words_)) != cudaSuccess) {
    cudaFree(words_);
    throw std::runtime_error("gpu_filter_data: cudaMemset failed");
  }
}

gpu_filter_data::~gpu_filter_data() { cudaFree(words_); }

}  // namespace adapter
}  // namespace dtlg
