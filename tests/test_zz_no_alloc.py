"""dtlg_batch_contains_noalloc: the probe for callers that cannot allocate.

Some callers cannot call cudaMalloc (their device memory belongs to their own
buffer manager or host application, or an allocation's synchronization is too
costly on their path).  This entry point keeps the probe's scratch in a static
device array instead; its results must equal the ordinary entry point's.
Checked through the C ABI on two calls in a row (the shared array keeps the
previous call's contents, so the second call shows that it is cleared), for
every filter kind (blocked Bloom, zoned Bloom, cuckoo, blocked cuckoo, classic
Bloom), plus the rejection of oversized calls.

Named test_zz_* so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import dtlg
import oracle as O
from dtlg import keygen

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MAX_KEYS = 1 << 26  # DTLG_NOALLOC_MAX_KEYS in include/dtlg.h


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def probe_existing(f, words, keys, offset):
    out = torch.full((max(1, keys.numel()),), -1, dtype=torch.int32, device="cuda")
    cnt = C.c_uint64(0)
    st = dtlg.lib().dtlg_batch_contains(f._h, _ptr(words), _ptr(keys), keys.numel(), _ptr(out),
                                        offset & 0xFFFFFFFF, C.byref(cnt), _stream())
    assert st == 0
    return out[:cnt.value].cpu().numpy().copy()


def probe_noalloc(f, words, keys, offset):
    out = torch.full((max(1, keys.numel()),), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    st = dtlg.lib().dtlg_batch_contains_noalloc(f._h, _ptr(words), _ptr(keys), keys.numel(), _ptr(out),
                                                offset & 0xFFFFFFFF, _ptr(cnt), _stream())
    assert st == 0, st
    torch.cuda.synchronize()
    n = int(cnt.item())
    assert 0 <= n <= keys.numel()
    return out[:n].cpu().numpy().copy()


def dev(keys):
    return torch.from_numpy(np.ascontiguousarray(keys, dtype=np.uint32).view(np.int32)).cuda()


def test_noalloc_bloom_matches_existing_entry_point_twice():
    m = 16 * 200000
    f = dtlg.bbf_64(m, 8, 8, 8)
    words = f.alloc_filter_data()
    assert f.batch_insert(words, dev(keygen.build_keys(200000, 41)))
    # first call: many tiles; second call: fewer keys, other offset and a key
    # pointer that is not 16-byte aligned, so stale scratch words would show
    k1 = dev(keygen.probe_keys(200000, 1_000_003, 0.3, 41)[0])
    k2 = dev(keygen.probe_keys(200000, 50_001, 0.6, 42)[0])[1:]
    for keys, off in ((k1, 5), (k2, (1 << 32) - 7)):
        ref = probe_existing(f, words, keys, off)
        got = probe_noalloc(f, words, keys, off)
        assert np.array_equal(got, ref)
    # and once more the first call, after the second
    assert np.array_equal(probe_noalloc(f, words, k1, 5), probe_existing(f, words, k1, 5))


def test_noalloc_cuckoo_matches_existing_entry_point_twice():
    m = 1 << 20
    f = dtlg.cf(m, 16, 4)
    oc = O.Cuckoo(16, 4, m)
    table = np.zeros(f.alloc_words(), dtype=np.uint64)
    oc.insert(table, keygen.build_keys(60000, 43))
    words = torch.from_numpy(table.view(np.int64)).cuda()
    for seed, n in ((43, 300_000), (44, 7)):
        keys = dev(keygen.probe_keys(60000, n, 0.4, seed)[0])
        assert np.array_equal(probe_noalloc(f, words, keys, 0), probe_existing(f, words, keys, 0))


@pytest.mark.parametrize("kind", ["zoned", "blocked_cuckoo", "classic"])
def test_noalloc_other_kinds_match_existing_entry_point_twice(kind):
    """The zoned, blocked cuckoo and classic kinds reach the same fused kernel
    with their own filter arguments; each is built on the GPU and probed twice
    in a row (a large call, then a small one from a misaligned key pointer)."""
    n = 80000
    if kind == "zoned":
        f = dtlg.zbbf_64(12 * n + 5, 8, 8, 4)
    elif kind == "blocked_cuckoo":
        f = dtlg.bcf(1 << 21, 64, 16, 4)
    else:
        f = dtlg.bloomfilter_logic(16 * n, 5, dtlg.MAGIC)
    words = f.alloc_filter_data()
    assert f.batch_insert(words, dev(keygen.build_keys(n, 45)))
    k1 = dev(keygen.probe_keys(n, 700_001, 0.25, 45)[0])
    k2 = dev(keygen.probe_keys(n, 33_333, 0.5, 46)[0])[3:]
    for keys, off in ((k1, 11), (k2, 0)):
        assert np.array_equal(probe_noalloc(f, words, keys, off), probe_existing(f, words, keys, off))


def test_noalloc_rejects_more_keys_than_its_scratch_serves():
    f = dtlg.bbf_32(1 << 16, 4)
    words = f.alloc_filter_data()
    keys = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    # key_cnt is only checked against the limit; nothing is launched or read
    st = dtlg.lib().dtlg_batch_contains_noalloc(f._h, _ptr(words), _ptr(keys), MAX_KEYS + 1, _ptr(out), 0,
                                                _ptr(cnt), _stream())
    assert st == 9  # DTLG_ERR_WORKSPACE
