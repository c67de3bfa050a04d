"""dtlg_sector_gather, the random-sector gather behind the L2 roofline of
bench.py, against a numpy restatement of its sector stream."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bloomfilter-bsd_b200"))

M64 = (1 << 64) - 1


def gather_rows(n, rows):
    """Row of sector i, for i < n (the hash the kernel documents)."""
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = i * np.uint64(0x9E3779B97F4A7C15)
        x ^= x >> np.uint64(29)
        x *= np.uint64(0xBF58476D1CE4E5B9)
        x ^= x >> np.uint64(32)
        return ((x & np.uint64(0xFFFFFFFF)) * np.uint64(rows)) >> np.uint64(32)


def expected_sink(words, n):
    rows = len(words) // 4
    r = gather_rows(n, rows).astype(np.int64)
    w = words.reshape(rows, 4)[r]
    with np.errstate(over="ignore"):
        mixed = w[:, 0] ^ (w[:, 1] * np.uint64(3)) ^ (w[:, 2] * np.uint64(5)) ^ (w[:, 3] * np.uint64(7))
    return int(np.bitwise_xor.reduce(mixed))


@pytest.mark.gpu
@pytest.mark.parametrize("mib,n", [(1, (1 << 20) + 37), (8, 1 << 22), (3, 4099)])
def test_sector_gather_matches_numpy(mib, n):
    import torch

    import dtlg

    rng = np.random.default_rng(mib * 1000 + n)
    words = rng.integers(0, 1 << 63, size=(mib << 20) // 8, dtype=np.uint64)
    d = torch.from_numpy(words.view(np.int64)).cuda()
    sink = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = dtlg.lib().dtlg_sector_gather(C.c_void_p(d.data_ptr()), mib << 20, n, C.c_void_p(sink.data_ptr()),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    got = int(sink.item()) & M64
    assert got == expected_sink(words, n)


def test_sector_gather_argument_errors():
    """Argument checks that return before any CUDA call (no GPU needed)."""
    import dtlg

    err_invalid_config, err_null, err_alignment = 1, 3, 4  # dtlg_status (include/dtlg.h)
    L = dtlg.lib()
    sink = C.c_uint64(0)
    assert L.dtlg_sector_gather(None, 1 << 20, 16, C.byref(sink), None) == err_null
    assert L.dtlg_sector_gather(C.c_void_p(64), 1 << 20, 16, None, None) == err_null
    assert L.dtlg_sector_gather(C.c_void_p(72), 1 << 20, 16, C.byref(sink), None) == err_alignment
    assert L.dtlg_sector_gather(C.c_void_p(64), 16, 16, C.byref(sink), None) == err_invalid_config
    assert L.dtlg_sector_gather(None, 1 << 20, 0, None, None) == 0
