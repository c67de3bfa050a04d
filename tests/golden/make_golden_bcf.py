"""Generate the blocked cuckoo filter golden vectors in tests/golden/ from the
reference itself.

Runs the reference's dtl::bcf (src/dtl/filter/bcf.cpp), compiled from its
sources by oracle/Makefile (``make -C oracle ref``) twice: for plain x86-64,
where every config takes the scalar batch path, and for AVX2, where <16,4> and
<8,4> take the SIMD batch path.  It needs the reference tree at build time
only; the fixtures it writes are committed and are all the tests need.

Contents of bcf_vectors.npz (index in bcf_index.json):
  * bcf_<i>_table: the filter words after the reference's batch_insert of the
    build keys (its kicks are random, so this table is one draw)
  * bcf_<i>_hits: the reference's scalar batch_contains match list over the
    probe keys; bcf_<i>_hits_avx2: the AVX2 build's list where it differs
Keys are regenerated from the seeds in bcf_index.json with dtlg.keygen.

    python tests/golden/make_golden_bcf.py
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

# (block bytes, tag bits, associativity): every tag/associativity pair, every
# block size; loads from light to overflowing.
BCF = [(64, 16, 4), (64, 8, 4), (64, 8, 8), (64, 10, 6), (64, 12, 4), (64, 16, 2),
       (8, 16, 4), (8, 8, 4), (32, 16, 2), (128, 12, 4), (256, 8, 8), (512, 16, 4), (512, 10, 6)]
BCF_M = (1 << 15, 20000)
LOADS = (0.5, 0.97)


def main():
    ref = O.RefBcf("scalar")
    ref_avx2 = O.RefBcf("avx2")
    arrays, index = {}, {"bcf": [], "invalid": []}
    i = 0
    for (bb, t, a) in BCF:
        for m in BCF_M:
            for load in LOADS:
                r = ref.create(m, bb, t, a)
                rv = ref_avx2.create(m, bb, t, a)
                assert r is not None and rv is not None, (bb, t, a, m)
                slots = (r.size_in_bytes * 8 // (t * a)) * a
                n_build = max(1, int(slots * load))
                seed = 7000 + i
                bk = keygen.build_keys(n_build, seed)
                data = r.alloc()
                r.insert(data, bk)
                pk, _ = keygen.probe_keys(n_build, 4000, 0.3, seed)
                hits = r.batch_contains(data, pk, 11 * i)
                hits_avx2 = rv.batch_contains(data, pk, 11 * i)
                arrays[f"bcf_{i}_table"] = data[: r.size_u32].copy()
                arrays[f"bcf_{i}_hits"] = hits
                if not np.array_equal(hits, hits_avx2):
                    arrays[f"bcf_{i}_hits_avx2"] = hits_avx2
                index["bcf"].append({"id": i, "block_bytes": bb, "t": t, "a": a, "m": m, "seed": seed,
                                     "n_build": n_build, "n_probe": 4000, "hit_ratio": 0.3,
                                     "match_offset": 11 * i, "name": r.name(), "size_u32": int(r.size_u32),
                                     "size_in_bytes": int(r.size_in_bytes),
                                     "avx2_differs": not np.array_equal(hits, hits_avx2)})
                i += 1
    # configurations the reference's constructor rejects (blocked_cuckoofilter.hpp:254-297)
    for (bb, t, a) in [(16, 16, 4), (1024, 16, 4), (64, 16, 8), (64, 4, 4), (64, 32, 1), (64, 12, 2)]:
        assert ref.create(1 << 15, bb, t, a) is None
        index["invalid"].append([bb, t, a])
    np.savez_compressed(os.path.join(HERE, "bcf_vectors.npz"), **arrays)
    with open(os.path.join(HERE, "bcf_index.json"), "w") as f:
        json.dump(index, f, indent=1)
    print(f"{len(index['bcf'])} blocked cuckoo fixtures")


if __name__ == "__main__":
    main()
