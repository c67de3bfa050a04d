"""Classic Bloom filter (dtl::bloomfilter_logic) on the CPU: the oracle
against the reference's own fixtures and, where oracle/_ref is built, against
the reference run live; the host-side configuration of libdtlg.so against the
oracle (no GPU calls)."""
import json
import os

import numpy as np
import pytest

import dtlg as F
import oracle as O
from dtlg import keygen

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def cbf_golden():
    d = os.path.join(HERE, "golden")
    with open(os.path.join(d, "cbf_index.json")) as f:
        index = json.load(f)
    return index, np.load(os.path.join(d, "cbf_vectors.npz"))


def test_oracle_matches_reference_fixtures(cbf_golden):
    index, arr = cbf_golden
    for e in index["cbf"]:
        o = O.ClassicBloom(e["k"], e["m"], e["magic"])
        assert o.word_cnt == e["size_u32"] and o.m_actual == e["m_actual"]
        bk = keygen.build_keys(e["n_build"], e["seed"])
        words = o.alloc()
        o.insert(words, bk)
        assert np.array_equal(words.view(np.uint32)[: o.word_cnt], arr[f"cbf_{e['id']}_words"]), e
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        assert np.array_equal(o.batch_contains(words, pk, e["match_offset"]), arr[f"cbf_{e['id']}_hits"]), e


def test_magic_bit_index_is_zero(cbf_golden):
    """As compiled, the reference's MAGIC classic filter sets bit 0 of each
    word only (its bit-index shift is out of range and folded to 0)."""
    index, arr = cbf_golden
    for e in index["cbf"]:
        if e["magic"] and e["k"] > 0:
            w = arr[f"cbf_{e['id']}_words"]
            assert np.all(w <= 1) and w.any()


def test_host_config_matches_oracle():
    for magic in (False, True):
        for k in (0, 1, 4, 17):
            for m in (0, 1, 32, 33, 1000, 1 << 20, 123457, 1 << 36):
                if magic and m == 1 << 36:
                    # 2^31 words: the next cheap MAGIC divisor exceeds 2^31 blocks
                    with pytest.raises(F.SizeError):
                        F.bloomfilter_logic(m, k, F.MAGIC)
                    with pytest.raises(ValueError):
                        O.ClassicBloom(k, m, True)
                    continue
                o = O.ClassicBloom(k, m, magic)
                f = F.bloomfilter_logic(m, k, F.MAGIC if magic else F.POWER_OF_TWO)
                assert f.block_cnt() == o.block_cnt and f.size_in_bytes() * 8 == o.m_actual
                assert f.size() == (o.word_cnt + 1) // 2 and f.is_magic() == magic
                assert f.kind() == "classic_bloom"
    with pytest.raises(F.InvalidConfig):
        F.bloomfilter_logic(1 << 20, 18)
    with pytest.raises(ValueError):
        O.ClassicBloom(18, 1 << 20)
    with pytest.raises(F.SizeError):
        F.bloomfilter_logic(1 << 37, 2)   # 2^32 words: more blocks than the addressing allows


ref = O.try_refcbf()


@pytest.mark.skipif(ref is None, reason="oracle/_ref/libdtlref_cbf.so not built")
def test_oracle_matches_reference_live():
    rng = np.random.default_rng(3)
    for magic in (False, True):
        for k in (0, 1, 2, 5, 8, 13, 17):
            for m in (33, 1000, 1 << 12, 100000, 3 << 20):
                o = O.ClassicBloom(k, m, magic)
                r = ref.create(k, m, magic)
                assert r.size_u32 == o.word_cnt and r.length == o.m_actual
                keys = rng.integers(0, 2**32, max(1, o.m_actual // (8 * max(k, 1))), dtype=np.uint32)
                d_r = r.alloc()
                assert r.insert(d_r, keys)
                d_o = o.alloc()
                o.insert(d_o, keys)
                assert np.array_equal(d_r[: r.size_u32], d_o.view(np.uint32)[: r.size_u32])
                probe = np.concatenate([keys[::2], rng.integers(0, 2**32, 10000, dtype=np.uint32)])
                assert np.array_equal(r.batch_contains(d_r, probe, 9), o.batch_contains(d_o, probe, 9))
    # more than 2^27 words: the POW2 bit shift wraps mod 32
    o = O.ClassicBloom(3, 1 << 33)
    r = ref.create(3, 1 << 33)
    keys = rng.integers(0, 2**32, 5000, dtype=np.uint32)
    d_r = r.alloc()
    r.insert(d_r, keys)
    d_o = o.alloc()
    o.insert(d_o, keys)
    assert np.array_equal(d_r[: r.size_u32], d_o.view(np.uint32)[: r.size_u32])
