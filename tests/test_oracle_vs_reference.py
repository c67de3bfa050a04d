"""The C restatement against the reference compiled from its sources
(oracle/_ref, built by ``make -C oracle ref``), over every config the
reference's dispatchers accept.  Skipped where the reference build is absent."""
import numpy as np
import pytest

import oracle as O
from gen_ref_instances import bloom_configs, cuckoo_configs

ref = O.try_reflib()
pytestmark = pytest.mark.skipif(ref is None, reason="oracle/_ref not built")


def test_all_bloom_configs_bit_exact():
    rng = np.random.default_rng(11)
    checked = 0
    for cfg in bloom_configs():
        for m in (1 << 14, (1 << 14) + 1000, 999):
            ob = O.Bloom(*cfg, m)
            r = ref.bloom(*cfg, m)
            if r is None:
                continue  # config not instantiated in this library variant
            assert r.word_cnt == ob.word_cnt and r.length == ob.m_actual
            if ob.block_cnt == 1 and not ob.magic:
                continue  # the reference shifts a u32 by 32 here (undefined)
            n = max(1, int(ob.m_actual // 16))
            keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
            d1, d2 = ob.alloc(), ob.alloc()
            r.insert(d1, keys)
            ob.insert(d2, keys)
            assert np.array_equal(d1, d2), cfg
            probe = np.concatenate([keys[: n // 4], rng.integers(0, 1 << 32, 2000, dtype=np.uint64)
                                    .astype(np.uint32)])
            assert np.array_equal(r.batch_contains(d1, probe, 5, unroll=0),
                                  ob.batch_contains(d1, probe, 5)), cfg
            checked += 1
    assert checked > 100


def test_all_cuckoo_configs_bit_exact():
    rng = np.random.default_rng(12)
    for (t, b) in cuckoo_configs():
        for m in (1 << 15, (1 << 15) + 999):
            oc = O.Cuckoo(t, b, m)
            r = ref.cuckoo(t, b, m)
            if r is None:
                continue
            keys = rng.integers(0, 1 << 32, int(oc.bucket_cnt * b * 0.7), dtype=np.uint64).astype(np.uint32)
            probe = np.concatenate([keys, rng.integers(0, 1 << 32, 5000, dtype=np.uint64).astype(np.uint32)])
            d = oc.alloc()
            r.insert(d, keys)               # the reference's own (random) build
            for u in (0, 1):
                assert np.array_equal(r.batch_contains(d, probe, 3, unroll=u), oc.batch_contains(d, probe, 3))
            assert r.count_occupied(d) == oc.count_occupied(d)
            d2 = oc.alloc()
            oc.insert(d2, keys, seed=9)     # the restatement's build, probed by the reference
            assert np.array_equal(r.batch_contains(d2, probe, 0), oc.batch_contains(d2, probe, 0))


def test_magic_matches_reference():
    rng = np.random.default_rng(13)
    for n in list(range(0, 300)) + [int(x) for x in rng.integers(2, 1 << 31, 300)]:
        assert ref.next_cheap_magic(n) == O.next_cheap_magic(n)
