// filter_handle.hpp -- the opaque dtlg_filter of include/dtlg.h.
#pragma once

#include "host_config.hpp"
#include "registry.hpp"

struct dtlg_filter {
  dtlg::FilterDesc d;
  const dtlg::BloomKernels* bk = nullptr;
  const dtlg::CuckooKernels* ck = nullptr;
};
