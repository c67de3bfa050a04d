"""Classic Bloom filter (dtl::bloomfilter_logic) on the GPU, through the C ABI:
byte-identical words after batch_insert and identical match lists against the
reference's own fixtures and the oracle, every probe plan."""
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


@pytest.fixture(scope="module")
def cbf_golden():
    d = os.path.join(HERE, "golden")
    with open(os.path.join(d, "cbf_index.json")) as f:
        index = json.load(f)
    return index, np.load(os.path.join(d, "cbf_vectors.npz"))


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


def test_reference_fixtures(cbf_golden):
    index, arr = cbf_golden
    for e in index["cbf"]:
        f = F.bloomfilter_logic(e["m"], e["k"], F.MAGIC if e["magic"] else F.POWER_OF_TWO)
        bk = keygen.build_keys(e["n_build"], e["seed"])
        w = f.alloc_filter_data()
        assert f.batch_insert(w, dev_keys(bk, pad=e["id"] % 4))
        got = w.cpu().numpy().view(np.uint32)[: e["size_u32"]]
        assert np.array_equal(got, arr[f"cbf_{e['id']}_words"]), e
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        for mode in (1, 2, 3, 4):
            f.set_probe_options(mode, e["id"] % 2)
            f.set_probe_passes(1 + e["id"] % 3)   # ignored: a classic probe is one pass
            assert np.array_equal(gpu_probe(f, w, pk, e["match_offset"], pad=(e["id"] + 1) % 4),
                                  arr[f"cbf_{e['id']}_hits"]), (e["id"], mode)


def test_large_filters_match_oracle():
    """8 MiB (L2-resident), 256 MiB and 1 GiB (2^28 words: the POW2 bit shift
    wraps) filters: GPU words equal the oracle's, probes of a sample agree."""
    for m, k, magic in ((1 << 26, 4, False), (1 << 31, 3, False), (3 << 29, 5, True), (1 << 33, 2, False)):
        o = O.ClassicBloom(k, m, magic)
        f = F.bloomfilter_logic(m, k, F.MAGIC if magic else F.POWER_OF_TWO)
        n = min(1 << 24, o.m_actual // (8 * k))
        bk = keygen.build_keys_torch(n, 77)
        w = f.alloc_filter_data()
        assert f.batch_insert(w, bk)
        words = w.cpu().numpy().view(np.uint64)
        ref = o.alloc()
        o.insert(ref, bk.cpu().numpy().view(np.uint32))
        assert np.array_equal(words, ref), (m, k, magic)
        pk, _ = keygen.probe_keys(n, 1 << 20, 0.2, 77)
        exp = o.batch_contains(ref, pk, 5)
        for mode in (1, 2, 4):   # 4 falls back to 2 above 192 KiB
            f.set_probe_options(mode, -1)
            assert np.array_equal(gpu_probe(f, w, pk, 5), exp), (m, k, magic, mode)
        del w, words, ref
        torch.cuda.empty_cache()
