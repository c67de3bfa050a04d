// ref_caldata_bridge.cpp -- C ABI over the reference's calibration-data file
// reader (model/calibration_data.cpp), its skyline lookup and its lookup-cost
// model (model/cost_fn.hpp), compiled from the reference's own sources
// (TEST INFRASTRUCTURE ONLY: it checks files written by dtlg.model.caldata).
#include <cstdint>
#include <cstring>
#include <string>

#include <dtl/filter/model/calibration_data.hpp>
#include <dtl/filter/model/cost_fn.hpp>

using dtl::filter::model::calibration_data;

namespace {
dtl::blocked_bloomfilter_config bbf(uint32_t k, uint32_t wb, uint32_t w, uint32_t s, uint32_t addr, uint32_t z) {
  dtl::blocked_bloomfilter_config c;
  c.k = k;
  c.word_size = wb;
  c.word_cnt_per_block = w;
  c.sector_cnt = s;
  c.addr_mode = addr ? dtl::block_addressing::MAGIC : dtl::block_addressing::POWER_OF_TWO;
  c.zone_cnt = z;
  return c;
}
}  // namespace

extern "C" {

uint64_t ref_cal_sizeof(int what) {
  switch (what) {
    case 0: return sizeof(dtl::blocked_bloomfilter_config);
    case 1: return sizeof(dtl::cuckoofilter::config);
    case 2: return sizeof(dtl::filter::model::timing);
    case 3: return sizeof(dtl::filter::model::tuning_params);
    case 4: return sizeof(dtl::filter::model::skyline_matrix::entry_t);
    default: return 0;
  }
}

void* ref_cal_open(const char* path) {
  try {
    return new calibration_data(std::string(path));
  } catch (...) {
    return nullptr;
  }
}

void ref_cal_close(void* h) { delete static_cast<calibration_data*>(h); }

uint64_t ref_cal_mem_levels(void* h) { return static_cast<calibration_data*>(h)->get_mem_levels(); }

uint64_t ref_cal_cache_size(void* h, uint32_t i) { return static_cast<calibration_data*>(h)->get_cache_sizes()[i]; }

uint64_t ref_cal_filter_size(void* h, uint32_t i) { return static_cast<calibration_data*>(h)->get_filter_sizes()[i]; }

uint64_t ref_cal_bbf_count(void* h) { return static_cast<calibration_data*>(h)->get_bbf_configs().size(); }

// delta t of one Bloom config at one memory level; returns 0 if unknown
int ref_cal_bbf_timing(void* h, uint32_t k, uint32_t wb, uint32_t w, uint32_t s, uint32_t addr, uint32_t z,
                       uint32_t level, double* cycles, double* nanos) {
  auto t = static_cast<calibration_data*>(h)->get_timings(bbf(k, wb, w, s, addr, z));
  if (level >= t.size()) return 0;
  *cycles = t[level].cycles_per_lookup;
  *nanos = t[level].nanos_per_lookup;
  return 1;
}

// cost_fn::lookup_costs(m, config, calibration_data) (cost_fn.hpp:131-141)
int ref_cal_lookup_cost(void* h, uint32_t k, uint32_t wb, uint32_t w, uint32_t s, uint32_t addr, uint32_t z,
                        uint64_t m, double* cycles, double* nanos) {
  try {
    auto t = dtl::filter::model::cost_fn::lookup_costs(m, bbf(k, wb, w, s, addr, z),
                                                        *static_cast<calibration_data*>(h));
    *cycles = t.cycles_per_lookup;
    *nanos = t.nanos_per_lookup;
    return 1;
  } catch (...) {
    return 0;
  }
}

// skyline_matrix::get_candidate_bbf_configs(n, tw)[0] (skyline_matrix.hpp:119-157)
int ref_cal_skyline(void* h, uint64_t n, uint64_t tw, uint32_t* cfg6, uint64_t* m, double* cycles) {
  const auto* sky = static_cast<calibration_data*>(h)->get_skyline_matrix();
  if (!sky) return 0;
  auto c = sky->get_candidate_bbf_configs(n, tw);
  if (c.empty()) return 0;
  const auto& e = c[0];
  cfg6[0] = e.config_.k;
  cfg6[1] = e.config_.word_size;
  cfg6[2] = e.config_.word_cnt_per_block;
  cfg6[3] = e.config_.sector_cnt;
  cfg6[4] = static_cast<uint32_t>(e.config_.addr_mode);
  cfg6[5] = e.config_.zone_cnt;
  *m = e.m_;
  *cycles = e.overhead_.cycles_per_lookup;
  return 1;
}

}  // extern "C"
