// filter_handle.hpp -- the opaque dtlg_filter of include/dtlg.h.
#pragma once

#include "host_config.hpp"
#include "registry.hpp"
#include "status.hpp"

struct dtlg_filter {
  dtlg::FilterDesc d;
  const dtlg::BloomKernels* bk = nullptr;
  const dtlg::CuckooKernels* ck = nullptr;
  const dtlg::BcfKernels* xk = nullptr;   // blocked cuckoo
  const dtlg::ClassicKernels* qk = nullptr;  // classic Bloom
  const dtlg::ProbeKernels* pk = nullptr;  // the probe kernels of whichever kind
  // probe tuning (dtlg_set_probe_options): mode 0 = auto, 1 = fused single
  // kernel, 2 = bitmask + compaction, 3 = partitioned, 4 = shared-memory
  // filter copy; bits_variant -1 = auto
  int probe_mode = 0;
  int bits_variant = -1;
  int probe_passes = 0;  // block-range passes of the two-pass probe; 0 = auto
  // Bloom build plan (dtlg_set_build_options): 0 = auto, 1 = one kernel of
  // global atomic ORs, 2 = keys grouped by block range first
  int build_mode = 0;
};

namespace dtlg {
// The filter fields of a probe launch.
inline void set_filter_args(const FilterDesc& d, ProbeArgs* a) {
  a->addr = d.addr;
  a->victim_word = d.victim_word;
  a->bcf_bucket_bits = d.bucket_bits;
  a->bcf_hash_shift = d.hash_shift;
  a->cbf_k = d.k;
  a->cbf_bit_shift = d.bit_shift;
  a->cbf_bit_mask = d.bit_mask;
}
}  // namespace dtlg
