// bcf_inst.cu -- compiled blocked cuckoo kernels for every tag size /
// associativity the reference's dispatcher accepts (blocked_cuckoofilter.hpp:
// 270-297); the block size is a run-time parameter of the kernels.
#include "registry.hpp"

namespace dtlg {
namespace {
struct RegBcf {
  RegBcf() {
    register_bcf(bcf_entry<8, 4>());
    register_bcf(bcf_entry<8, 8>());
    register_bcf(bcf_entry<10, 6>());
    register_bcf(bcf_entry<12, 4>());
    register_bcf(bcf_entry<16, 2>());
    register_bcf(bcf_entry<16, 4>());
  }
} reg_bcf;
}  // namespace
}  // namespace dtlg
