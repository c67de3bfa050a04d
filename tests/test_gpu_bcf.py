"""Blocked cuckoo filter (dtl::bcf) on the GPU, through the C ABI.

Probe: bit-exact against the reference's own fixtures (tables built by the
reference, match lists from its scalar batch path) and against the oracle, in
every probe plan.  Build: the reference's build is randomised (kicks), so the
GPU build is checked by invariants -- no false negatives, the probe of the
GPU-built table equal to the oracle's probe of the same table, the same
per-bucket tag sets as a sequential build when no bucket fills up, and a false
positive rate close to the oracle build's.
"""
import json
import os

import numpy as np
import pytest

import dtlg as F
import oracle as O
from dtlg import keygen

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
TAG_PAIRS = [(8, 4), (8, 8), (10, 6), (12, 4), (16, 2), (16, 4)]
BLOCKS = [8, 32, 64, 128, 256, 512]


@pytest.fixture(scope="module")
def bcf_golden():
    d = os.path.join(HERE, "golden")
    with open(os.path.join(d, "bcf_index.json")) as f:
        index = json.load(f)
    return index, np.load(os.path.join(d, "bcf_vectors.npz"))


def dev_keys(keys, pad=0):
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    buf = torch.zeros(len(k) + 8, dtype=torch.int32, device="cuda")
    if len(k):
        buf[pad:pad + len(k)] = torch.from_numpy(k.view(np.int32)).cuda()
    return buf[pad:pad + len(k)]


def gpu_probe(f, words_t, keys, offset=0, pad=0):
    kt = dev_keys(keys, pad)
    out = torch.full((max(1, len(keys)),), -1, dtype=torch.int32, device="cuda")
    n = f.batch_contains(words_t, kt, len(keys), out, offset)
    return out[:n].cpu().numpy().view(np.uint32).copy()


def upload(f, table_u32):
    w = f.alloc_filter_data()
    t = np.zeros(w.numel() * 2, dtype=np.uint32)
    t[: len(table_u32)] = table_u32
    w.copy_(torch.from_numpy(t.view(np.int64)))
    return w


def host64(words_t):
    return words_t.cpu().numpy().view(np.uint64).copy()


def test_probe_reference_fixtures(bcf_golden):
    index, arr = bcf_golden
    for e in index["bcf"]:
        f = F.bcf(e["m"], e["block_bytes"], e["t"], e["a"])
        w = upload(f, arr[f"bcf_{e['id']}_table"])
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        exp = arr[f"bcf_{e['id']}_hits"]
        for mode in (1, 2, 3):
            f.set_probe_options(mode, e["id"] % 2)
            f.set_probe_passes(1 + e["id"] % 3)
            got = gpu_probe(f, w, pk, e["match_offset"], pad=e["id"] % 4)
            assert np.array_equal(got, exp), (e["id"], mode)


def test_probe_filter_not_32_byte_aligned(bcf_golden):
    """A filter base that is 16- but not 32-byte aligned takes the word-load
    path instead of the 256-bit sector loads; results are the same."""
    index, arr = bcf_golden
    for e in index["bcf"][::3]:
        f = F.bcf(e["m"], e["block_bytes"], e["t"], e["a"])
        n64 = f.alloc_words()
        buf = torch.zeros(n64 + 4, dtype=torch.int64, device="cuda")
        w = buf[2:2 + n64]
        assert w.data_ptr() % 32 == 16
        t = np.zeros(n64 * 2, dtype=np.uint32)
        t[: len(arr[f"bcf_{e['id']}_table"])] = arr[f"bcf_{e['id']}_table"]
        w.copy_(torch.from_numpy(t.view(np.int64)))
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        for mode in (1, 2, 3):
            f.set_probe_options(mode, -1)
            got = gpu_probe(f, w, pk, e["match_offset"])
            assert np.array_equal(got, arr[f"bcf_{e['id']}_hits"]), (e["id"], mode)


def test_build_invariants_every_config():
    for ci, (bb, (t, a)) in enumerate([(bb, ta) for bb in BLOCKS for ta in TAG_PAIRS]):
        for m in (1 << 17, 100003):
            o = O.BlockedCuckoo(m, bb, t, a)
            f = F.bcf(m, bb, t, a)
            slots = (o.m_actual // (t * a)) * a
            n = int(slots * (0.95 if ci % 2 else 0.6))
            seed = 300 + ci
            bk = keygen.build_keys(n, seed)
            w = f.alloc_filter_data()
            assert f.batch_insert(w, dev_keys(bk, pad=ci % 4))
            words = host64(w)
            # no false negatives, seen by the oracle and by the GPU
            assert len(o.batch_contains(words, bk)) == n, (bb, t, a, m)
            pk, _ = keygen.probe_keys(n, 5000, 0.2, seed)
            exp = o.batch_contains(words, pk, 3)
            for mode in (1, 2, 3):
                f.set_probe_options(mode, -1)
                assert np.array_equal(gpu_probe(f, w, pk, 3, pad=(ci + 1) % 4), exp), (bb, t, a, m, mode)
            assert len(gpu_probe(f, w, bk)) == n


def _bucket_sets(o, words, t, a):
    wb = o.word_bytes
    x = words.view(np.uint32 if wb == 4 else np.uint64)
    full = (1 << t) - 1
    tags = [(x >> np.array(t * j, dtype=x.dtype)) & np.array(full, dtype=x.dtype) for j in range(a)]
    return np.sort(np.stack(tags, axis=1), axis=1)


def test_light_build_same_tag_sets_as_sequential():
    """When no bucket can fill up, every key lands in its first bucket in any
    insertion order: the GPU build then holds the same tags per bucket as the
    oracle's sequential build.  Keys are kept only if each of their two
    buckets is a candidate bucket of at most `a` keys."""
    from collections import Counter
    for bb, (t, a) in [(64, (16, 4)), (64, (8, 8)), (512, (10, 6)), (32, (16, 2)), (128, (12, 4)), (8, (8, 4))]:
        m = 1 << 20
        o = O.BlockedCuckoo(m, bb, t, a)
        f = F.bcf(m, bb, t, a)
        keys = keygen.build_keys(int((o.m_actual // (t * a)) * a * 0.05), 17)
        loc = [o.locate(k) for k in keys]
        cnt = Counter()
        for blk, b1, b2, _ in loc:
            cnt[(blk, b1)] += 1
            if b2 != b1:
                cnt[(blk, b2)] += 1
        bk = np.array([k for k, (blk, b1, b2, _) in zip(keys, loc)
                       if cnt[(blk, b1)] <= a and cnt[(blk, b2)] <= a], dtype=np.uint32)
        assert len(bk) > 0.5 * len(keys)
        ref = o.alloc()
        o.insert(ref, bk, seed=1)
        w = f.alloc_filter_data()
        f.batch_insert(w, dev_keys(bk))
        got = host64(w)
        assert np.array_equal(_bucket_sets(o, got, t, a), _bucket_sets(o, ref, t, a)), (bb, t, a)


def test_fpr_matches_oracle_build():
    m = 1 << 24
    for bb, (t, a) in [(64, (16, 4)), (64, (8, 4)), (256, (12, 4))]:
        o = O.BlockedCuckoo(m, bb, t, a)
        f = F.bcf(m, bb, t, a)
        n = int((o.m_actual // (t * a)) * a * 0.85)
        bk = keygen.build_keys(n, 23)
        ref = o.alloc()
        o.insert(ref, bk, seed=2)
        w = f.alloc_filter_data()
        f.batch_insert(w, dev_keys(bk))
        neg = keygen.build_keys(1 << 20, 23, start=n)  # non-members (seeded bijection)
        fp_gpu = len(gpu_probe(f, w, neg))
        fp_ref = len(o.batch_contains(ref, neg))
        # the concurrent build interleaves relocation chains, so overflow marks
        # (which answer every key of a bucket) may differ a little in number:
        # within 25 % + 5 sigma of the sequential build's count
        tol = 0.25 * fp_ref + 5 * np.sqrt(fp_ref + 1)
        assert abs(fp_gpu - fp_ref) <= tol, (bb, t, a, fp_gpu, fp_ref)


def test_large_partitioned_probe():
    """A 256 MiB filter (DRAM-resident): the partitioned and the bitmask plans
    agree, a random subset agrees with the oracle, no false negatives."""
    m = 1 << 31
    f = F.bcf(m, 64, 16, 4)
    o = O.BlockedCuckoo(m, 64, 16, 4)
    n = 1 << 24
    bk = keygen.build_keys_torch(n, 41)
    w = f.alloc_filter_data()
    assert f.batch_insert(w, bk)
    pk, _ = keygen.probe_keys_torch(n, 1 << 25, 0.1, 41)
    out = torch.empty(1 << 25, dtype=torch.int32, device="cuda")
    res = {}
    for mode in (2, 3):
        f.set_probe_options(mode, -1)
        c = f.batch_contains(w, pk, pk.numel(), out, 0)
        res[mode] = out[:c].cpu().numpy().copy()
    assert np.array_equal(res[2], res[3])
    words = host64(w)
    sub = pk[: 1 << 18].cpu().numpy().view(np.uint32)
    exp = o.batch_contains(words, sub)
    assert np.array_equal(res[3][res[3] < (1 << 18)].view(np.uint32), exp)
    f.set_probe_options(3, -1)
    assert f.batch_contains(w, bk, n, out, 0) == n


def test_partitioned_build():
    """Build plan 2 (keys grouped by block range first, on request): the same
    invariants as the one-kernel build, and a false positive rate like it."""
    for bb, (t, a) in [(64, (16, 4)), (512, (10, 6)), (8, (8, 4)), (128, (12, 4))]:
        m = (1 << 22) + 4096 * (bb % 3)
        o = O.BlockedCuckoo(m, bb, t, a)
        f = F.bcf(m, bb, t, a)
        n = int((o.m_actual // (t * a)) * a * 0.8)
        bk = keygen.build_keys(n, 51)
        f.set_build_options(2)
        w = f.alloc_filter_data()
        assert f.batch_insert(w, dev_keys(bk, pad=1))
        words = host64(w)
        assert len(o.batch_contains(words, bk)) == n, (bb, t, a)
        pk, _ = keygen.probe_keys(n, 20000, 0.2, 51)
        assert np.array_equal(gpu_probe(f, w, pk, 9), o.batch_contains(words, pk, 9)), (bb, t, a)
    # 256 MiB: plan 2 against plan 1
    m = 1 << 31
    f = F.bcf(m, 64, 16, 4)
    n = 1 << 25
    bk = keygen.build_keys_torch(n, 52)
    neg = keygen.build_keys_torch(1 << 22, 52, start=n)
    out = torch.empty(max(n, 1 << 22), dtype=torch.int32, device="cuda")
    fps = []
    for mode in (2, 1):
        f.set_build_options(mode)
        w = f.alloc_filter_data()
        assert f.batch_insert(w, bk)
        assert f.batch_contains(w, bk, n, out, 0) == n
        fps.append(f.batch_contains(w, neg, neg.numel(), out, 0))
        del w
        torch.cuda.empty_cache()
    assert abs(fps[0] - fps[1]) <= 0.25 * fps[1] + 5 * np.sqrt(fps[1] + 1), fps


def test_partitioned_build_with_overflowing_range():
    """Blocked cuckoo keys skewed into one 8 MiB range overflow its segment of
    the partition; those keys come from the exact spill list (a second insert
    of a cuckoo key would take a second slot): every key placed once, no
    false negatives, the GPU's probe of the table equal to the oracle's."""
    m = 1 << 31                                   # 256 MiB, 64-byte blocks: 32 ranges of 2^17 blocks
    o = O.BlockedCuckoo(m, 64, 16, 4)
    f = F.bcf(m, 64, 16, 4)
    c1 = 370248451                                # the blocked cuckoo's block hash constant
    out, start = [], 0
    while sum(len(x) for x in out) < 1 << 20:
        k = keygen.build_keys(1 << 23, 81, start=start)
        start += 1 << 23
        out.append(k[((k.astype(np.uint64) * np.uint64(c1)) & np.uint64(0xFFFFFFFF)) < np.uint64(1 << 27)])
    bk = np.concatenate(out)[: 1 << 20]          # all in range 0: a quarter of its slots
    f.set_build_options(2)
    w = f.alloc_filter_data()
    assert f.batch_insert(w, dev_keys(bk))
    f.set_build_options(0)
    words = host64(w)
    assert len(o.batch_contains(words, bk)) == len(bk)
    pk = np.concatenate([bk[::7], keygen.build_keys(100000, 82, start=1 << 30)])
    assert np.array_equal(gpu_probe(f, w, pk, 3), o.batch_contains(words, pk, 3))
