"""The C restatement (oracle/dtl_oracle.c) against the reference's own
known-answer test and the golden vectors produced by the reference itself
(tests/golden/make_golden.py)."""
import numpy as np
import pytest

import oracle as O
from dtlg import keygen


def test_reference_known_answer():
    # src/dtl/filter/filter_test.cpp:16-40: default config (k=8, 4-byte word,
    # w=1, s=1), m=1024; keys {13,37,42,88} -> [0,1,2,3];
    # probe {0,1,42,2} with match_offset 1000 -> exactly [1002].
    f = O.Bloom(4, 1, 1, 1, 8, 1024)
    d = f.alloc()
    f.insert(d, [13, 37, 42, 88])
    assert f.batch_contains(d, [13, 37, 42, 88], 0).tolist() == [0, 1, 2, 3]
    assert f.batch_contains(d, [0, 1, 42, 2], 1000).tolist() == [1002]


def test_kat_words_match_reference(golden):
    index, arr = golden
    kat = index["kat"][0]
    f = O.Bloom(*kat["cfg"], kat["m"])
    d = f.alloc()
    f.insert(d, kat["build"])
    assert np.array_equal(d, arr["kat_words"])
    assert kat["hits1"] == [0, 1, 2, 3] and kat["hits2"] == [1002]


def test_next_cheap_magic_golden(golden):
    _, arr = golden
    for n, d, m, s in zip(arr["magic_n"], arr["magic_d"], arr["magic_m"], arr["magic_s"]):
        assert O.next_cheap_magic(int(n)) == (int(d), int(m), int(s)), n


def test_fast_mod_property():
    # test/div_test.cpp:11-40: a % d == fast_mod_u32(a, next_cheap_magic(b))
    rng = np.random.default_rng(3)
    L = O.lib()
    for b in rng.integers(1, (1 << 32) - 3, 200):
        d, mg, sh = O.next_cheap_magic(int(b))
        for a in rng.integers(0, 1 << 32, 50):
            assert L.orc_fast_mod(int(a), d, mg, sh) == int(a) % d


def test_bloom_golden(golden):
    index, arr = golden
    differs = set()
    for e in index["bloom"]:
        f = O.Bloom(*e["cfg"], e["m"])
        assert f.word_cnt == e["word_cnt"] and f.m_actual == e["m_actual"], e
        bk = keygen.build_keys(e["n_build"], e["seed"])
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        d = f.alloc()
        f.insert(d, bk)
        assert np.array_equal(d, arr[f"bloom_{e['id']}_words"]), e
        hits = f.batch_contains(d, pk, e["match_offset"])
        assert np.array_equal(hits, arr[f"bloom_{e['id']}_hits"]), e
        if e["simd_differs"]:
            differs.add(tuple(e["cfg"]))
    # The reference's SIMD and scalar paths disagree exactly where its unrolled
    # k=8 word block leaves a stale hash value behind: two words of k/w = 8
    # (w=2, k=16) or two zones of k/z = 8 (z=2, k=16).
    assert differs == {c for c in map(tuple, (e["cfg"] for e in index["bloom"]))
                       if c[4] == 16 and ((c[3] == 1 and c[1] == 2) or c[3] == 2)}


def test_cuckoo_golden(golden):
    index, arr = golden
    for e in index["cuckoo"]:
        f = O.Cuckoo(e["t"], e["b"], e["m"])
        assert f.s_.m_actual == e["m_actual"]
        table = arr[f"cuckoo_{e['id']}_table"]
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        hits = f.batch_contains(table, pk, e["match_offset"])
        assert np.array_equal(hits, arr[f"cuckoo_{e['id']}_hits"]), e
        assert f.count_occupied(table) == e["occupied"]


@pytest.mark.parametrize("cfg", [(4, 1, 1, 1, 0), (4, 3, 1, 1, 4), (4, 1, 2, 1, 1), (4, 1, 8, 1, 8),
                                 (4, 1, 1, 1, 17), (4, 2, 4, 1, 6), (4, 4, 4, 4, 8), (4, 8, 8, 2, 7),
                                 (4, 2, 2, 2, 8), (8, 8, 8, 16, 16), (2, 1, 1, 1, 4)])
def test_invalid_bloom_configs_rejected(cfg):
    with pytest.raises(ValueError):
        O.Bloom(*cfg, 1 << 16)


def test_sizes():
    # MAGIC vs POW2 chosen by whether m is a power of two (blocked_bloomfilter.hpp:234-242)
    f = O.Bloom(8, 8, 8, 1, 8, 1 << 20)
    assert not f.magic and f.block_cnt == (1 << 20) // 512
    g = O.Bloom(8, 8, 8, 1, 8, 3 * (1 << 19))
    assert g.magic and g.block_cnt >= 3 * (1 << 19) // 512
    c = O.Cuckoo(16, 4, 1 << 20)
    assert c.bucket_cnt == (1 << 20) // 64 and c.size_u64 == (1 << 20) // 64
