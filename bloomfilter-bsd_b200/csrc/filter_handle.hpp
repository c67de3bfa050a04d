// filter_handle.hpp -- the opaque dtlg_filter of include/dtlg.h.
#pragma once

#include "host_config.hpp"
#include "registry.hpp"
#include "status.hpp"

struct dtlg_filter {
  dtlg::FilterDesc d;
  const dtlg::BloomKernels* bk = nullptr;
  const dtlg::CuckooKernels* ck = nullptr;
  // probe tuning (dtlg_set_probe_options): mode 0 = auto, 1 = fused single
  // kernel, 2 = bitmask + compaction; bits_variant -1 = auto
  int probe_mode = 0;
  int bits_variant = -1;
  int probe_passes = 0;  // block-range passes of the two-pass probe; 0 = auto
};
