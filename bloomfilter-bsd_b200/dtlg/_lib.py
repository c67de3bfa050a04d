"""ctypes binding of libdtlg.so (include/dtlg.h).

The product path: every filter operation in this package goes through these
entry points into the sm_100a kernels.  There is no CPU fallback: if the
library is missing, importing the package raises.
"""
import ctypes as C
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("DTLG_LIB", os.path.join(PKG_ROOT, "lib", "libdtlg.so"))

OK = 0
STATUS = {
    0: "ok", 1: "invalid configuration", 2: "filter size out of range", 3: "null pointer",
    4: "filter words must be 16-byte aligned", 5: "CUDA error", 6: "allocation failed",
    7: "cuckoo filter full", 8: "device wait timed out", 9: "workspace too small",
    10: "unsupported operation",
}


class DtlgError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = STATUS.get(status, f"status {status}")
        if status == 5:
            msg += ": " + lib().dtlg_last_cuda_error().decode()
        super().__init__(f"{what}: {msg}" if what else msg)


class InvalidConfig(DtlgError, ValueError):
    """The reference's std::invalid_argument (blocked_bloomfilter.hpp:111)."""


class SizeError(DtlgError, ValueError):
    """The reference's std::logic_error on block counts (block_addressing_logic.hpp:81)."""


class BloomConfigS(C.Structure):
    _fields_ = [("k", C.c_uint32), ("word_size", C.c_uint32), ("word_cnt_per_block", C.c_uint32),
                ("sector_cnt", C.c_uint32), ("addr_mode", C.c_uint32), ("zone_cnt", C.c_uint32)]


class CuckooConfigS(C.Structure):
    _fields_ = [("bits_per_tag", C.c_uint32), ("tags_per_bucket", C.c_uint32), ("addr_mode", C.c_uint32)]


class BcfConfigS(C.Structure):
    _fields_ = [("block_size_bytes", C.c_uint32), ("tag_size_bits", C.c_uint32), ("associativity", C.c_uint32)]


class ClassicConfigS(C.Structure):
    _fields_ = [("k", C.c_uint32), ("addr_mode", C.c_uint32)]


class BatchItemS(C.Structure):
    _fields_ = [("filter", C.c_void_p), ("filter_words", C.c_void_p), ("build_keys", C.c_void_p),
                ("n_build", C.c_uint32), ("probe_keys", C.c_void_p), ("n_probe", C.c_uint32),
                ("match_positions", C.c_void_p), ("match_offset", C.c_uint32), ("match_cnt", C.c_void_p)]


class ProbePlanS(C.Structure):
    _fields_ = [("mode", C.c_int), ("variant", C.c_int), ("passes", C.c_int), ("ms", C.c_float),
                ("gkeys_per_s", C.c_float)]


class BatchPlanS(C.Structure):
    _fields_ = [("staging", C.c_int), ("ctas_per_sm", C.c_int), ("ms", C.c_float)]


class CostTablesS(C.Structure):
    _fields_ = [("n_cand", C.c_uint32), ("n_bpk", C.c_uint32), ("bits_per_key", C.c_void_p), ("fpr", C.c_void_p),
                ("n_size", C.c_uint32), ("log2_bytes_first", C.c_double), ("log2_bytes_step", C.c_double),
                ("ns_per_key", C.c_void_p), ("ns_per_match", C.c_double), ("l2_budget_bytes", C.c_double),
                ("ns_second", C.c_void_p)]


class CostQueryS(C.Structure):
    _fields_ = [("log2_n", C.c_double), ("fpr_target", C.c_double), ("hit_ratio", C.c_double),
                ("work_ns", C.c_double), ("l2_resident", C.c_uint32)]


# every entry point declared in include/dtlg.h: name -> (restype, argtypes)
_vp, _u32, _u64, _i = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
_u64p = C.POINTER(C.c_uint64)
SIGNATURES = {
    "dtlg_bloom_create": (_i, [C.POINTER(BloomConfigS), _u64, C.POINTER(_vp)]),
    "dtlg_cuckoo_create": (_i, [C.POINTER(CuckooConfigS), _u64, C.POINTER(_vp)]),
    "dtlg_blocked_cuckoo_create": (_i, [C.POINTER(BcfConfigS), _u64, C.POINTER(_vp)]),
    "dtlg_classic_bloom_create": (_i, [C.POINTER(ClassicConfigS), _u64, C.POINTER(_vp)]),
    "dtlg_destroy": (None, [_vp]),
    "dtlg_size_in_bytes": (_u64, [_vp]),
    "dtlg_size": (_u64, [_vp]),
    "dtlg_alloc_words_u64": (_u64, [_vp]),
    "dtlg_name": (C.c_size_t, [_vp, C.c_char_p, C.c_size_t]),
    "dtlg_kind": (_i, [_vp]),
    "dtlg_block_cnt": (_u64, [_vp]),
    "dtlg_is_magic": (_i, [_vp]),
    "dtlg_batch_insert": (_i, [_vp, _vp, _vp, _u32, _u64p, _vp]),
    "dtlg_batch_contains": (_i, [_vp, _vp, _vp, _u32, _vp, _u32, _u64p, _vp]),
    "dtlg_batch_contains_async": (_i, [_vp, _vp, _vp, _u32, _vp, _u32, _vp, _vp]),
    "dtlg_probe_workspace_size": (C.c_size_t, [_u32]),
    "dtlg_batch_contains_ws": (_i, [_vp, _vp, _vp, _u32, _vp, _u32, _vp, _vp, C.c_size_t, _vp]),
    "dtlg_batch_contains_gather": (_i, [_vp, _vp, _vp, _u32, _u32, _vp, _vp, _vp, _vp, _u32, _vp, _vp, C.c_size_t,
                                        _vp]),
    "dtlg_batch_contains_noalloc": (_i, [_vp, _vp, _vp, _u32, _vp, _u32, _vp, _vp]),
    "dtlg_set_probe_options": (_i, [_vp, _i, _i]),
    "dtlg_set_probe_passes": (_i, [_vp, _i]),
    "dtlg_set_build_options": (_i, [_vp, _i]),
    "dtlg_probe_kernel_count": (_i, [_vp, _u32]),
    "dtlg_set_l2_fetch_granularity": (_i, [_i, C.POINTER(_i)]),
    "dtlg_autotune_probe": (_i, [_vp, _vp, _vp, _u32, _vp, _i, _vp, C.POINTER(ProbePlanS)]),
    "dtlg_batch_autotune": (_i, [_vp, _i, _vp, C.POINTER(BatchPlanS)]),
    "dtlg_batch_set_staging": (_i, [_vp, _i]),
    "dtlg_batch_staged_count": (_u32, [_vp]),
    "dtlg_batch_prepare": (_i, [C.POINTER(BatchItemS), _u32, _i, C.POINTER(_vp)]),
    "dtlg_batch_run": (_i, [_vp, _vp]),
    "dtlg_batch_set_ctas_per_sm": (_i, [_vp, _i]),
    "dtlg_batch_kernel_count": (_i, [_vp]),
    "dtlg_batch_fallback_count": (_u32, [_vp]),
    "dtlg_batch_destroy": (None, [_vp]),
    "dtlg_cost_search": (_i, [C.POINTER(CostTablesS), _vp, _u32, _vp, _vp, _vp, _vp, _vp, _i]),
    "dtlg_cost_eval": (_i, [C.POINTER(CostTablesS), _vp, _u32, _vp, _vp, _vp]),
    "dtlg_mlp_create": (_i, [_u32, _u32, _u32, _u32, _u32, C.POINTER(_vp)]),
    "dtlg_mlp_destroy": (None, [_vp]),
    "dtlg_mlp_param_count": (_u64, [_vp]),
    "dtlg_mlp_set_params": (_i, [_vp, _vp]),
    "dtlg_mlp_get_params": (_i, [_vp, _vp]),
    "dtlg_mlp_get_grads": (_i, [_vp, _vp]),
    "dtlg_mlp_forward": (_i, [_vp, _vp, _u32, _vp, _vp]),
    "dtlg_mlp_loss_grad": (_i, [_vp, _vp, _vp, _vp, _u32, _vp, _vp]),
    "dtlg_mlp_adam_step": (_i, [_vp, C.c_float, C.c_float, C.c_float, C.c_float, _vp]),
    "dtlg_mlp_train": (_i, [_vp, _vp, _vp, _vp, _u32, _vp, _u32, _u32, C.c_float, C.c_float, _vp, _vp]),
    "dtlg_mlp_choose": (_i, [_vp, _vp, _u32, _u32, _vp, _vp, _vp, _vp]),
    "dtlg_or_words": (_i, [_vp, _vp, _u64, _u32, _u64, _vp]),
    "dtlg_copy_words_peer": (_i, [_vp, C.c_int, _vp, C.c_int, _u64, _vp]),
    "dtlg_sector_gather": (_i, [_vp, _u64, _u64, _vp, _vp]),
    "dtlg_check_wait_timeout": (_i, [_u32, C.POINTER(_u32)]),
    "dtlg_insert": (_i, [_vp, _vp, _u32, _vp]),
    "dtlg_contains": (_i, [_vp, _vp, _u32, C.POINTER(_i), _vp]),
    "dtlg_batch_contains_host": (_i, [_vp, _vp, _vp, _u64, _vp, _u32, _u64p, _vp]),
    "dtlg_batch_insert_host": (_i, [_vp, _vp, _vp, _u64, _u64p, _vp]),
    "dtlg_count_occupied_slots": (_i, [_vp, _vp, _u64p, _vp]),
    "dtlg_status_string": (C.c_char_p, [_i]),
    "dtlg_last_cuda_error": (C.c_char_p, []),
    "dtlg_version": (C.c_char_p, []),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libdtlg.so not built at {LIB_PATH} (make -C bloomfilter-bsd_b200)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, what=""):
    if status == OK:
        return
    if status == 1:
        raise InvalidConfig(status, what)
    if status == 2:
        raise SizeError(status, what)
    raise DtlgError(status, what)
