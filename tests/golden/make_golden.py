"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own filter logic, compiled from its sources into
oracle/_ref/libdtlref_avx512.so by oracle/Makefile (``make -C oracle ref``).
It needs the reference tree at build time only; the fixtures it writes are
committed and are all the tests need afterwards.

Contents of reference_vectors.npz (index in index.json):
  * magic_n/_d/_m/_s: dtl::next_cheap_magic(n) (div.hpp:30-57) for a spread of n
  * bloom_<i>_words/_hits/_hits_simd: filter words after the reference's
    batch_insert of build keys, and its batch_contains match lists (scalar
    path, and the SIMD path for the configs where the two differ)
  * cuckoo_<i>_table/_hits: a table built by the reference's (randomised)
    insert and its batch_contains match list over probe keys
Keys are regenerated from the seeds in index.json with dtlg.keygen.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "bloomfilter-bsd_b200"))

import oracle as O  # noqa: E402
from dtlg import keygen  # noqa: E402

# (word bytes, w, s, z, k): register-blocked, sectorized (sgew), sltw and zoned
# layouts, including the k=16 configs whose SIMD and scalar paths disagree.
BLOOM = [
    (4, 1, 1, 1, 8), (4, 1, 1, 1, 4), (4, 1, 4, 1, 8), (8, 1, 1, 1, 1), (8, 1, 8, 1, 8),
    (8, 1, 2, 1, 6), (4, 2, 2, 1, 16), (8, 2, 4, 1, 16), (4, 2, 2, 1, 6), (4, 4, 4, 1, 4),
    (8, 8, 8, 1, 8), (8, 8, 16, 1, 16), (4, 16, 16, 1, 16), (8, 4, 4, 1, 12), (4, 8, 8, 1, 8),
    (4, 16, 1, 1, 4), (8, 8, 1, 1, 8), (4, 8, 2, 1, 6), (8, 16, 4, 1, 8), (4, 4, 1, 1, 3),
    (8, 4, 2, 1, 10), (4, 16, 8, 1, 16), (8, 2, 1, 1, 7), (8, 8, 8, 2, 8), (8, 8, 8, 4, 8),
    (4, 16, 16, 2, 8), (4, 16, 16, 4, 8), (4, 8, 8, 2, 16), (8, 16, 16, 8, 16), (4, 4, 4, 2, 6),
    (8, 4, 4, 2, 16), (8, 16, 16, 2, 16),
]
BLOOM_M = (1 << 13, 10000)
CUCKOO = [(t, b) for t in (4, 8, 12, 16, 32) for b in (1, 2, 4)]
CUCKOO_M = (1 << 14, 12000)


def main():
    ref = O.RefLib("avx512")
    arrays, index = {}, {"bloom": [], "cuckoo": [], "kat": []}

    rng = np.random.default_rng(20241203)
    ns = sorted(set([0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 100, 127, 128,
                     129, 1000, 1023, 1024, 1025, (1 << 16) - 1, 1 << 16, (1 << 16) + 1,
                     (1 << 20) + 7, (1 << 24) - 3, (1 << 30) + 1, (1 << 31) - 1, 1 << 31,
                     17660000, 4415056, 1103764]
                    + [int(x) for x in rng.integers(2, 1 << 31, 160)]))
    mags = [ref.next_cheap_magic(n) for n in ns]
    arrays["magic_n"] = np.array(ns, dtype=np.uint64)
    arrays["magic_d"] = np.array([x[0] for x in mags], dtype=np.uint32)
    arrays["magic_m"] = np.array([x[1] for x in mags], dtype=np.uint32)
    arrays["magic_s"] = np.array([x[2] for x in mags], dtype=np.uint32)

    i = 0
    for cfg in BLOOM:
        for m in BLOOM_M:
            r = ref.bloom(*cfg, m)
            assert r is not None, (cfg, m)
            words = r.word_cnt
            word_bytes = cfg[0]
            data = np.zeros(max(1, (words * word_bytes + 7) // 8), dtype=np.uint64)
            n_build = max(1, (r.length // 12))
            seed = 1000 + i
            bk = keygen.build_keys(n_build, seed)
            r.insert(data, bk)
            pk, _ = keygen.probe_keys(n_build, 3000, 0.3, seed)
            hits = r.batch_contains(data, pk, 1000 + i, unroll=0)
            hits_simd = r.batch_contains(data, pk, 1000 + i, unroll=1)
            arrays[f"bloom_{i}_words"] = data
            arrays[f"bloom_{i}_hits"] = hits
            if not np.array_equal(hits, hits_simd):
                arrays[f"bloom_{i}_hits_simd"] = hits_simd
            index["bloom"].append({"id": i, "cfg": list(cfg), "m": m, "seed": seed, "n_build": int(n_build),
                                   "n_probe": 3000, "hit_ratio": 0.3, "match_offset": 1000 + i,
                                   "word_cnt": int(words), "m_actual": int(r.length),
                                   "simd_differs": not np.array_equal(hits, hits_simd)})
            i += 1

    j = 0
    for (t, b) in CUCKOO:
        for m in CUCKOO_M:
            r = ref.cuckoo(t, b, m)
            oc = O.Cuckoo(t, b, m)
            data = oc.alloc()
            n_build = int(oc.bucket_cnt * b * 0.8)
            seed = 5000 + j
            bk = keygen.build_keys(n_build, seed)
            ok = r.insert(data, bk)
            pk, _ = keygen.probe_keys(n_build, 3000, 0.3, seed)
            hits = r.batch_contains(data, pk, 7 * j, unroll=1)
            assert np.array_equal(hits, r.batch_contains(data, pk, 7 * j, unroll=0))
            arrays[f"cuckoo_{j}_table"] = data
            arrays[f"cuckoo_{j}_hits"] = hits
            index["cuckoo"].append({"id": j, "t": t, "b": b, "m": m, "seed": seed, "n_build": n_build,
                                    "n_probe": 3000, "hit_ratio": 0.3, "match_offset": 7 * j,
                                    "insert_ok": bool(ok), "m_actual": int(r.length),
                                    "occupied": int(r.count_occupied(data))})
            j += 1

    # The reference's known-answer test, run through the reference:
    # src/dtl/filter/filter_test.cpp:16-40 (default blocked_bloomfilter_config,
    # k=8, 4-byte words, w=1, s=1, m=1024).
    r = ref.bloom(4, 1, 1, 1, 8, 1024)
    data = np.zeros((r.word_cnt * 4 + 7) // 8, dtype=np.uint64)
    r.insert(data, np.array([13, 37, 42, 88], dtype=np.uint32))
    index["kat"].append({
        "cfg": [4, 1, 1, 1, 8], "m": 1024, "build": [13, 37, 42, 88],
        "probe1": [13, 37, 42, 88], "offset1": 0,
        "hits1": r.batch_contains(data, np.array([13, 37, 42, 88], dtype=np.uint32), 0).tolist(),
        "probe2": [0, 1, 42, 2], "offset2": 1000,
        "hits2": r.batch_contains(data, np.array([0, 1, 42, 2], dtype=np.uint32), 1000).tolist()})
    arrays["kat_words"] = data

    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **arrays)
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1)
    print(f"{len(index['bloom'])} bloom, {len(index['cuckoo'])} cuckoo fixtures, {len(ns)} magic values")


if __name__ == "__main__":
    main()
