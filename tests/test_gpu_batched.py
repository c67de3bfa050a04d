"""The batched multi-filter build+probe (one persistent kernel) against the
oracle: every filter's words and ascending match positions must equal the
per-filter result."""
import numpy as np
import pytest

import dtlg as F
import oracle as O
from dtlg import keygen
from dtlg.batch import Batch, BatchItem

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MENU = [(8, 8, 8, 1, 8), (8, 8, 8, 2, 8), (8, 8, 8, 4, 8), (4, 16, 16, 2, 8), (4, 16, 16, 4, 8), (4, 1, 1, 1, 4),
        (4, 1, 1, 1, 8)]
OTHER = [(8, 4, 4, 1, 4), (4, 16, 1, 1, 4), (8, 2, 2, 1, 16)]   # not in the compiled menu: separate launches


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def make_batch(rng, n_filters):
    cases = []
    for i in range(n_filters):
        cfg = (MENU + OTHER)[i % (len(MENU) + len(OTHER))]
        n_build = int(rng.choice([0, 1, 5, 1000, 4096, 4097, int(2 ** rng.uniform(10, 17))]))
        n_probe = int(rng.choice([0, 3, 4096, 8191, int(2 ** rng.uniform(12, 18))]))
        bpk = int(rng.choice([8, 12, 16]))
        m = max(64, n_build * bpk) + (i % 3) * 777
        cases.append((cfg, m, n_build, n_probe, 1000 * i))
    return cases


@pytest.mark.parametrize("use_graph", [True, False])
def test_batched_matches_oracle(use_graph):
    rng = np.random.default_rng(5 if use_graph else 6)
    cases = make_batch(rng, 40)
    items, refs = [], []
    for i, (cfg, m, nb, npb, off) in enumerate(cases):
        wb, w, s, z, k = cfg
        f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                     zone_cnt=z), m)
        ob = O.Bloom(wb, w, s, z, k, m)
        bk = keygen.build_keys(nb, 900 + i)
        pk, _ = keygen.probe_keys(nb, npb, 0.3, 900 + i)
        rw = ob.alloc()
        ob.insert(rw, bk)
        refs.append((rw, ob.batch_contains(rw, pk, off)))
        items.append(BatchItem(f, f.alloc_filter_data(), dev(bk), dev(pk),
                               torch.full((max(1, npb),), -1, dtype=torch.int32, device="cuda"),
                               torch.full((1,), -1, dtype=torch.int64, device="cuda"), off))
    b = Batch(items, use_graph=use_graph)
    assert b.fallback_count() == sum(1 for c in cases if c[0] in OTHER)
    for rep in range(3):  # later runs (graph replays) must not see earlier queue / status words
        for it in items:
            it.filter_data.zero_()
        b.run()
        torch.cuda.synchronize()
        for (rw, exp), it, c in zip(refs, items, cases):
            assert np.array_equal(it.filter_data.cpu().numpy().view(np.uint64), rw), (c, rep)
            n = int(it.match_cnt.item())
            assert n == len(exp), (c, rep)
            assert np.array_equal(it.match_positions[:n].cpu().numpy().view(np.uint32), exp), (c, rep)


def test_batched_ctas_per_sm_tuning_keeps_results():
    rng = np.random.default_rng(7)
    cases = [((8, 8, 8, 2, 8), 200000 * 12 + 5, 200000, 300000, 0), ((4, 1, 1, 1, 4), 1 << 20, 60000, 100000, 7)]
    items, refs = [], []
    for i, (cfg, m, nb, npb, off) in enumerate(cases):
        f = F.construct(F.blocked_bloomfilter_config(k=cfg[4], word_size=cfg[0], word_cnt_per_block=cfg[1],
                                                     sector_cnt=cfg[2], zone_cnt=cfg[3]), m)
        ob = O.Bloom(*cfg, m)
        bk = keygen.build_keys(nb, 50 + i)
        pk, _ = keygen.probe_keys(nb, npb, 0.05, 50 + i)
        rw = ob.alloc()
        ob.insert(rw, bk)
        refs.append(ob.batch_contains(rw, pk, off))
        items.append(BatchItem(f, f.alloc_filter_data(), dev(bk), dev(pk),
                               torch.zeros(npb, dtype=torch.int32, device="cuda"),
                               torch.zeros(1, dtype=torch.int64, device="cuda"), off))
    b = Batch(items)
    assert b.kernel_count() == 1
    for cps in (1, 2, 0):
        b.set_ctas_per_sm(cps)
        for it in items:
            it.filter_data.zero_()
        b.run()
        torch.cuda.synchronize()
        for exp, it in zip(refs, items):
            n = int(it.match_cnt.item())
            assert np.array_equal(it.match_positions[:n].cpu().numpy().view(np.uint32), exp)
