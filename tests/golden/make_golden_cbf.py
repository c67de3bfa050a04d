"""Generate the classic Bloom filter golden vectors in tests/golden/ from the
reference itself.

Runs the reference's dtl::bloomfilter_logic<uint32_t, A>
(src/dtl/filter/bloomfilter/bloomfilter_logic.hpp), compiled from its header
by oracle/Makefile (``make -C oracle ref`` -> oracle/_ref/libdtlref_cbf.so).
It needs the reference tree at build time only; the fixtures it writes are
committed and are all the tests need.

Contents of cbf_vectors.npz (index in cbf_index.json):
  * cbf_<i>_words: the filter words after the reference's batch_insert
  * cbf_<i>_hits: its batch_contains match list over the probe keys
Keys are regenerated from the seeds in cbf_index.json with dtlg.keygen.

    python tests/golden/make_golden_cbf.py
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

# (k, m bits, MAGIC?): POW2 and MAGIC, k from 0 to 17, sizes from two words on
# (a single POW2 word makes the reference index word h >> 32: out of bounds)
CBF = [(k, m, magic) for k in (0, 1, 2, 3, 4, 6, 8, 11, 16, 17)
       for (m, magic) in (((1 << 14), False), (64, False), (20000, True), (33, True))]


def main():
    ref = O.RefCbf()
    arrays, index = {}, {"cbf": []}
    for i, (k, m, magic) in enumerate(CBF):
        r = ref.create(k, m, magic)
        assert r is not None
        n_build = max(1, r.length // (8 * max(k, 1)))
        seed = 9000 + i
        bk = keygen.build_keys(n_build, seed)
        words = r.alloc()
        assert r.insert(words, bk)
        pk, _ = keygen.probe_keys(n_build, 3000, 0.3, seed)
        arrays[f"cbf_{i}_words"] = words[: r.size_u32].copy()
        arrays[f"cbf_{i}_hits"] = r.batch_contains(words, pk, 13 * i)
        index["cbf"].append({"id": i, "k": k, "m": m, "magic": magic, "seed": seed, "n_build": int(n_build),
                             "n_probe": 3000, "hit_ratio": 0.3, "match_offset": 13 * i,
                             "size_u32": int(r.size_u32), "m_actual": int(r.length)})
    np.savez_compressed(os.path.join(HERE, "cbf_vectors.npz"), **arrays)
    with open(os.path.join(HERE, "cbf_index.json"), "w") as f:
        json.dump(index, f, indent=1)
    print(f"{len(index['cbf'])} classic Bloom fixtures")


if __name__ == "__main__":
    main()
