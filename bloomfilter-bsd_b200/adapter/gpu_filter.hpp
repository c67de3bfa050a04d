// gpu_filter.hpp -- the drop-in on the reference's side: a dtl::filter::filter_base
// (src/dtl/filter/filter_base.hpp:11-62) whose members forward to libdtlg.so's
// C ABI (include/dtlg.h), so the reference's callers -- its filter facade,
// model::benchmark, user code holding a filter_base* -- build and probe on the
// GPU without a change of code.
//
// Differences from the CPU filters, all forced by the device:
//  * filter_data, keys and match_positions are DEVICE pointers (as every
//    non-_host entry point of the ABI); gpu_filter_data allocates the words
//    (the facade's filter_shared allocates a NUMA vector instead,
//    filter.hpp:113-119);
//  * work goes to the stream given at construction (0: the legacy default
//    stream); batch_contains blocks until the count is known, as the
//    reference's call returns it;
//  * a CUDA failure throws std::runtime_error (the reference's members cannot
//    fail); construction throws std::invalid_argument / std::logic_error where
//    the reference's constructors do (DTLG_ERR_INVALID_CONFIG / DTLG_ERR_SIZE).
//
// Build: g++ -std=c++14 -I<reference>/src -I<reference> -Iinclude, link
// -ldtlg -lcudart.  The reference's headers include one Boost.Align header;
// where Boost is not installed, adapter/boost_compat supplies that one name.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include <dtl/filter/filter_base.hpp>

#include "dtlg.h"

namespace dtlg {
namespace adapter {

// Throws the exception the reference throws for the same condition.
void throw_status(dtlg_status st, const char* what);

class gpu_filter : public dtl::filter::filter_base {
 public:
  // bbf_32 / bbf_64 / zbbf_32 / zbbf_64 by config (filter.hpp:42-72): word
  // size 4 or 8, zone_cnt 1 = blocked / sectorized, > 1 = zoned.
  gpu_filter(const dtlg_bloom_config& config, std::size_t m, cudaStream_t stream = nullptr);
  // cf(m, bits_per_tag, tags_per_bucket) (cf.hpp, filter.hpp:168-169)
  gpu_filter(const dtlg_cuckoo_config& config, std::size_t m, cudaStream_t stream = nullptr);
  ~gpu_filter() override;
  gpu_filter(gpu_filter&& o) noexcept;
  gpu_filter& operator=(gpu_filter&& o) noexcept;
  // the base's move-assignment (noexcept): only from another gpu_filter
  dtl::filter::filter_base& operator=(dtl::filter::filter_base&& o) noexcept override;

  $u1 insert(word_t* __restrict filter_data, key_t key) override;
  $u1 batch_insert(word_t* __restrict filter_data, const key_t* __restrict keys, u32 key_cnt) override;
  $u1 contains(const word_t* __restrict filter_data, key_t key) const override;
  $u64 batch_contains(const word_t* __restrict filter_data, const key_t* __restrict keys, u32 key_cnt,
                      $u32* __restrict match_positions, u32 match_offset) const override;
  std::string name() const override;
  std::size_t size_in_bytes() const override;
  std::size_t size() const override;

  // 64-bit words to allocate on the device: size(), plus for cuckoo filters
  // the victim record the reference keeps past size() (cuckoofilter_logic.hpp:
  // 145-157) and read slack.
  std::size_t alloc_words() const;
  const dtlg_filter* handle() const { return f_; }

 private:
  dtlg_filter* f_ = nullptr;
  cudaStream_t stream_ = nullptr;
};

// Zeroed device memory for a gpu_filter's words (the counterpart of the
// facade's filter_data vector, filter.hpp:92-119).
class gpu_filter_data {
 public:
  explicit gpu_filter_data(const gpu_filter& f);
  ~gpu_filter_data();
  gpu_filter_data(const gpu_filter_data&) = delete;
  gpu_filter_data& operator=(const gpu_filter_data&) = delete;
  dtl::filter::filter_base::word_t* data() { return words_; }
  std::size_t words() const { return n_; }

 private:
  dtl::filter::filter_base::word_t* words_ = nullptr;
  std::size_t n_ = 0;
};

}  // namespace adapter
}  // namespace dtlg
