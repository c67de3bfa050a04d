"""Blocked cuckoo filter (dtl::bcf) on the CPU: the oracle against the
reference's own fixtures and, where oracle/_ref is built, against the reference
run live; the host-side configuration of libdtlg.so against the reference's
sizes, names and rejected configs (no GPU calls)."""
import json
import os

import numpy as np
import pytest

import dtlg as F
import oracle as O
from dtlg import keygen

HERE = os.path.dirname(os.path.abspath(__file__))
TAG_PAIRS = [(8, 4), (8, 8), (10, 6), (12, 4), (16, 2), (16, 4)]
BLOCKS = [8, 32, 64, 128, 256, 512]


@pytest.fixture(scope="module")
def bcf_golden():
    d = os.path.join(HERE, "golden")
    with open(os.path.join(d, "bcf_index.json")) as f:
        index = json.load(f)
    return index, np.load(os.path.join(d, "bcf_vectors.npz"))


def _table64(table_u32):
    t = np.ascontiguousarray(table_u32, dtype=np.uint32)
    if len(t) % 2:
        t = np.concatenate([t, np.zeros(1, dtype=np.uint32)])
    return t.view(np.uint64).copy()


def test_oracle_matches_reference_fixtures(bcf_golden):
    index, arr = bcf_golden
    for e in index["bcf"]:
        o = O.BlockedCuckoo(e["m"], e["block_bytes"], e["t"], e["a"])
        assert o.size_u32 == e["size_u32"]
        data = _table64(arr[f"bcf_{e['id']}_table"])
        bk = keygen.build_keys(e["n_build"], e["seed"])
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        assert np.array_equal(o.batch_contains(data, pk, e["match_offset"]), arr[f"bcf_{e['id']}_hits"]), e
        # the reference's build has no false negatives
        assert len(o.batch_contains(data, bk)) == e["n_build"]


def test_host_config_matches_reference(bcf_golden):
    index, _ = bcf_golden
    for e in index["bcf"]:
        f = F.bcf(e["m"], e["block_bytes"], e["t"], e["a"])
        assert f.name() == e["name"]
        assert f.size_in_bytes() == e["size_in_bytes"]
        assert 2 * f.size() == e["size_u32"]
        assert f.kind() == "blocked_cuckoo"
    for bb, t, a in index["invalid"]:
        with pytest.raises(F.InvalidConfig):
            F.bcf(1 << 15, bb, t, a)
        with pytest.raises(ValueError):
            O.BlockedCuckoo(1 << 15, bb, t, a)


def test_host_config_matches_oracle_sweep():
    for bb in BLOCKS:
        for t, a in TAG_PAIRS:
            for m in (0, 1, 64, 511, 1 << 12, 1 << 20, 123457, 3 << 20, 1 << 30):
                o = O.BlockedCuckoo(m, bb, t, a)
                f = F.bcf(m, bb, t, a)
                assert f.block_cnt() == o.block_cnt and f.is_magic() == o.magic
                assert 2 * f.size() == o.size_u32 and f.size_in_bytes() * 8 == o.m_actual


def test_size_limit():
    # 32-bit word indexes (blocked_cuckoofilter_logic.hpp:76): 2^32 words at most
    F.bcf(1 << 37, 8, 16, 4)                     # 2^31 blocks of one u64 word
    with pytest.raises(F.SizeError):
        F.bcf(1 << 38, 8, 16, 4)                 # 2^32 blocks
    with pytest.raises(F.SizeError):
        F.bcf(1 << 38, 512, 16, 2)               # 2^26 blocks x 128 u32 words = 2^33 words
    with pytest.raises(ValueError):
        O.BlockedCuckoo(1 << 38, 8, 16, 4)


def test_avx2_batch_path_superset(bcf_golden):
    """The reference's AVX2 batch path of <16,4> and <8,4> reports the scalar
    matches plus keys whose bucket holds an all-ones tag field
    (blocked_cuckoofilter_simd.hpp: per-field overflow compare); the GPU kernel
    follows the scalar path."""
    index, arr = bcf_golden
    seen = 0
    for e in index["bcf"]:
        if not e["avx2_differs"]:
            continue
        assert (e["t"], e["a"]) in ((16, 4), (8, 4))
        seen += 1
        o = O.BlockedCuckoo(e["m"], e["block_bytes"], e["t"], e["a"])
        data = _table64(arr[f"bcf_{e['id']}_table"])
        words = data.view(np.uint32 if o.word_bytes == 4 else np.uint64)
        wpb = e["block_bytes"] // o.word_bytes
        scalar, avx2 = arr[f"bcf_{e['id']}_hits"], arr[f"bcf_{e['id']}_hits_avx2"]
        assert np.all(np.isin(scalar, avx2))
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        full = (1 << e["t"]) - 1
        for pos in np.setdiff1d(avx2, scalar):
            blk, b1, b2, _ = o.locate(pk[pos - e["match_offset"]])
            fields = [(int(words[blk * wpb + b]) >> (e["t"] * j)) & full for b in (b1, b2) for j in range(e["a"])]
            assert full in fields
    assert seen > 0


def test_oracle_build_no_false_negatives():
    rng = np.random.default_rng(5)
    for bb in BLOCKS:
        for t, a in TAG_PAIRS:
            for m in (1 << 16, 50000):
                o = O.BlockedCuckoo(m, bb, t, a)
                slots = (o.m_actual // (t * a)) * a
                keys = rng.integers(0, 2**32, int(slots * 0.9), dtype=np.uint32)
                data = o.alloc()
                o.insert(data, keys, seed=3)
                assert len(o.batch_contains(data, keys)) == len(keys)


ref = O.try_refbcf("scalar")


@pytest.mark.skipif(ref is None, reason="oracle/_ref/libdtlref_bcf.so not built")
def test_oracle_matches_reference_live():
    rng = np.random.default_rng(11)
    for bb in BLOCKS:
        for t, a in TAG_PAIRS:
            for m in (1 << 18, 77777):
                o = O.BlockedCuckoo(m, bb, t, a)
                r = ref.create(m, bb, t, a)
                assert r.size_u32 == o.size_u32 and r.name() == F.bcf(m, bb, t, a).name()
                keys = rng.integers(0, 2**32, int(o.m_actual / (t * 1.6)), dtype=np.uint32)
                probe = np.concatenate([keys[::3], rng.integers(0, 2**32, 20000, dtype=np.uint32)])
                data = r.alloc()
                r.insert(data, keys)
                d64 = _table64(data[: r.size_u32])
                assert np.array_equal(r.batch_contains(data, probe, 5), o.batch_contains(d64, probe, 5))
                # oracle-built table, probed by the reference
                d2 = o.alloc()
                o.insert(d2, keys, seed=9)
                d2r = np.zeros(r.size_u32 + 16, dtype=np.uint32)
                d2r[: r.size_u32] = d2.view(np.uint32)[: r.size_u32]
                assert np.array_equal(r.batch_contains(d2r, probe, 1), o.batch_contains(d2, probe, 1))
