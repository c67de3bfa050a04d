// cuckoo_inst.cu -- compiled cuckoo kernels for every tag size / associativity
// the reference's dispatcher accepts (cuckoofilter.hpp:184-206).
#include "registry.hpp"

namespace dtlg {
namespace {
struct RegCuckoo {
  RegCuckoo() {
    register_cuckoo(cuckoo_entry<4, 1>());
    register_cuckoo(cuckoo_entry<4, 2>());
    register_cuckoo(cuckoo_entry<4, 4>());
    register_cuckoo(cuckoo_entry<8, 1>());
    register_cuckoo(cuckoo_entry<8, 2>());
    register_cuckoo(cuckoo_entry<8, 4>());
    register_cuckoo(cuckoo_entry<12, 1>());
    register_cuckoo(cuckoo_entry<12, 2>());
    register_cuckoo(cuckoo_entry<12, 4>());
    register_cuckoo(cuckoo_entry<16, 1>());
    register_cuckoo(cuckoo_entry<16, 2>());
    register_cuckoo(cuckoo_entry<16, 4>());
    register_cuckoo(cuckoo_entry<32, 1>());
    register_cuckoo(cuckoo_entry<32, 2>());
    register_cuckoo(cuckoo_entry<32, 4>());
  }
} reg_cuckoo;
}  // namespace
}  // namespace dtlg
