"""Failure detection of the bounded device waits, without a GPU fault.

dtlg_check_wait_timeout runs the look-back wait of the ordered compaction and
the batched kernel's dependency wait against words that nothing sets, with a
short spin limit: both must give up, set their error bits and let the kernel
end; the context must stay usable (a probe right after it is bit-exact)."""
import ctypes as C
import os
import sys
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "bloomfilter-bsd_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

ERR_INVALID_CONFIG, ERR_NULL = 1, 3  # dtlg_status (include/dtlg.h)


@pytest.mark.gpu
@pytest.mark.parametrize("limit", [1, 1000, 20000])
def test_waits_give_up_and_report(limit):
    import torch

    import dtlg
    import oracle as O
    from dtlg import keygen

    torch.cuda.set_device(0)
    bits = C.c_uint32(0)
    t0 = time.perf_counter()
    assert dtlg.lib().dtlg_check_wait_timeout(limit, C.byref(bits)) == 0
    assert time.perf_counter() - t0 < 30
    assert bits.value == 3  # look-back (bit 0) and dependency wait (bit 1) both reported

    # the context is still usable: a probe (bitmask plan, with the look-back of
    # its compaction) right after it, bit-exact against the oracle
    m = 16 * 50000
    g = dtlg.bbf_64(m, 8, 8, 8)
    ob = O.Bloom(8, 8, 8, 1, 8, m)
    bk = keygen.build_keys(50000, 4)
    words = g.alloc_filter_data("cuda:0")
    assert g.batch_insert(words, torch.from_numpy(bk.view(np.int32)).cuda(0))
    ref = ob.alloc()
    ob.insert(ref, bk)
    pk, _ = keygen.probe_keys(50000, 1 << 21, 0.2, 4)
    out = torch.empty(1 << 21, dtype=torch.int32, device="cuda:0")
    n = g.batch_contains(words, torch.from_numpy(pk.view(np.int32)).cuda(0), 1 << 21, out, 0)
    exp = ob.batch_contains(ref, pk, 0)
    assert n == len(exp) and np.array_equal(out[:n].cpu().numpy().view(np.uint32), exp)


def test_wait_check_argument_errors():
    """Argument checks that return before any CUDA call (no GPU needed)."""
    import dtlg

    L = dtlg.lib()
    bits = C.c_uint32(0)
    assert L.dtlg_check_wait_timeout(100, None) == ERR_NULL
    assert L.dtlg_check_wait_timeout(0, C.byref(bits)) == ERR_INVALID_CONFIG
    assert L.dtlg_check_wait_timeout((1 << 22) + 1, C.byref(bits)) == ERR_INVALID_CONFIG
