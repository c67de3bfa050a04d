"""Many filters built and probed in one persistent kernel (dtlg_batch_* ABI).

No counterpart in the reference, where each filter of a query plan is built
and probed by its own filter_base::batch_insert / batch_contains calls
(filter_base.hpp:26,42-45).  A Batch holds the device tables of such a list of
calls; run() executes all of them as one persistent kernel, by default
replayed as a CUDA graph.  The tensors named by the items must stay alive and
in place for the lifetime of the Batch.
"""
import ctypes as C
from dataclasses import dataclass

from . import _lib
from ._lib import check, lib
from .filter import _dev_ptr, _stream


@dataclass
class BatchItem:
    filter: object          # a dtlg filter_base (Bloom)
    filter_data: object     # CUDA int64 tensor, zeroed for a fresh build
    build_keys: object      # CUDA int32 tensor
    probe_keys: object      # CUDA int32 tensor
    match_positions: object  # CUDA int32 tensor, >= len(probe_keys)
    match_cnt: object       # CUDA int64 tensor of 1 element
    match_offset: int = 0


class Batch:
    def __init__(self, items, use_graph=True):
        self.items = list(items)
        arr = (_lib.BatchItemS * max(1, len(self.items)))()
        for i, it in enumerate(self.items):
            arr[i] = _lib.BatchItemS(
                it.filter._h, _dev_ptr(it.filter_data, "filter_data"),
                _dev_ptr(it.build_keys, "build_keys") if it.build_keys.numel() else None, it.build_keys.numel(),
                _dev_ptr(it.probe_keys, "probe_keys") if it.probe_keys.numel() else None, it.probe_keys.numel(),
                _dev_ptr(it.match_positions, "match_positions"), int(it.match_offset) & 0xFFFFFFFF,
                _dev_ptr(it.match_cnt, "match_cnt"))
        h = C.c_void_p()
        check(lib().dtlg_batch_prepare(arr, len(self.items), int(bool(use_graph)), C.byref(h)), "batch_prepare")
        self._h = h

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                lib().dtlg_batch_destroy(h)
            except Exception:
                pass

    def run(self):
        check(lib().dtlg_batch_run(self._h, _stream()), "batch_run")

    def set_ctas_per_sm(self, n):
        check(lib().dtlg_batch_set_ctas_per_sm(self._h, int(n)), "batch_set_ctas_per_sm")

    def autotune(self, reps=3):
        """Times every (staging, CTAs per SM) choice and keeps the fastest;
        returns {"staging", "ctas_per_sm", "ms"}."""
        plan = _lib.BatchPlanS()
        check(lib().dtlg_batch_autotune(self._h, int(reps), _stream(), C.byref(plan)), "batch_autotune")
        return {"staging": plan.staging, "ctas_per_sm": plan.ctas_per_sm, "ms": plan.ms}

    def set_staging(self, staging):
        """0: build filters of up to 64 MiB range by range in shared memory
        (default); 1: global atomic inserts only.  Results are identical."""
        check(lib().dtlg_batch_set_staging(self._h, int(staging)), "batch_set_staging")

    def staged_count(self):
        return lib().dtlg_batch_staged_count(self._h)

    def kernel_count(self):
        return lib().dtlg_batch_kernel_count(self._h)

    def fallback_count(self):
        return lib().dtlg_batch_fallback_count(self._h)
