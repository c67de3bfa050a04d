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


@pytest.mark.parametrize("use_graph,staging", [(True, 0), (False, 0), (True, 1)])
def test_batched_matches_oracle(use_graph, staging):
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
    b.set_staging(staging)
    assert b.fallback_count() == sum(1 for c in cases if c[0] in OTHER)
    assert (b.staged_count() > 0) == (staging == 0)
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


def test_staged_build_with_skewed_keys_overflows_exactly():
    """Keys that all fall into a few ranges overflow their buckets; the rest
    of those keys takes the direct path and the words still match."""
    rng = np.random.default_rng(8)
    items, refs = [], []
    for i, cfg in enumerate([(8, 8, 8, 1, 8), (8, 8, 8, 2, 8), (4, 16, 16, 4, 8), (4, 1, 1, 1, 4)]):
        wb, w, s, z, k = cfg
        n = 300000
        few = keygen.build_keys(5, 70 + i)
        bk = np.concatenate([np.repeat(few, n // 10), keygen.build_keys(n // 2, 80 + i)])
        bk = bk[rng.permutation(len(bk))].astype(np.uint32)
        m = (n * 12) | 1
        f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                     zone_cnt=z), m)
        ob = O.Bloom(wb, w, s, z, k, m)
        rw = ob.alloc()
        ob.insert(rw, bk)
        pk = np.concatenate([few, keygen.probe_keys(n, 50000, 0.2, 90 + i)[0]]).astype(np.uint32)
        refs.append((rw, ob.batch_contains(rw, pk, 3)))
        items.append(BatchItem(f, f.alloc_filter_data(), dev(bk), dev(pk),
                               torch.zeros(len(pk), dtype=torch.int32, device="cuda"),
                               torch.zeros(1, dtype=torch.int64, device="cuda"), 3))
    b = Batch(items)
    assert b.staged_count() == len(items)
    for _ in range(2):
        for it in items:
            it.filter_data.zero_()
        b.run()
        torch.cuda.synchronize()
        for (rw, exp), it in zip(refs, items):
            assert np.array_equal(it.filter_data.cpu().numpy().view(np.uint64), rw)
            n = int(it.match_cnt.item())
            assert np.array_equal(it.match_positions[:n].cpu().numpy().view(np.uint32), exp)


def test_staged_build_ors_into_existing_words():
    """batch_insert ORs into the caller's words: a staged build over a filter
    that already holds keys equals building both key sets."""
    wb, w, s, z, k = (8, 8, 8, 2, 8)
    m = 1 << 22
    f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                 zone_cnt=z), m)
    ob = O.Bloom(wb, w, s, z, k, m)
    a, c = keygen.build_keys(100000, 1), keygen.build_keys(200000, 2)
    rw = ob.alloc()
    ob.insert(rw, a)
    data = torch.from_numpy(rw.copy().view(np.int64)).cuda()
    ob.insert(rw, c)
    pk = keygen.probe_keys(100000, 10000, 0.5, 1)[0]
    item = BatchItem(f, data, dev(c), dev(pk), torch.zeros(len(pk), dtype=torch.int32, device="cuda"),
                     torch.zeros(1, dtype=torch.int64, device="cuda"), 0)
    b = Batch([item], use_graph=False)
    assert b.staged_count() == 1
    b.run()
    torch.cuda.synchronize()
    assert np.array_equal(data.cpu().numpy().view(np.uint64), rw)


def test_batch_with_blocked_cuckoo_and_classic_filters():
    """Blocked cuckoo and classic Bloom filters join a batch as separate
    launches (the persistent kernel's menu holds the blocked Bloom layouts):
    classic words byte-identical to the oracle's, blocked cuckoo words probed
    by the oracle to the same match list, no false negatives; the Bloom
    filters of the batch still go through the persistent kernel."""
    items, checks = [], []
    specs = [("bloom", 20000), ("bcf", 30000), ("classic", 25000), ("bloom", 5000), ("bcf", 3000)]
    for i, (kind, nb) in enumerate(specs):
        bk = keygen.build_keys(nb, 60 + i)
        pk, _ = keygen.probe_keys(nb, 3 * nb, 0.3, 60 + i)
        if kind == "bloom":
            f = F.construct(F.blocked_bloomfilter_config(k=8, word_size=8, word_cnt_per_block=8, sector_cnt=8), nb * 12)
            o = O.Bloom(8, 8, 8, 1, 8, nb * 12)
        elif kind == "bcf":
            f = F.bcf(nb * 32 + 11, 64, 16, 4)
            o = O.BlockedCuckoo(nb * 32 + 11, 64, 16, 4)
        else:
            f = F.bloomfilter_logic(nb * 10, 4)
            o = O.ClassicBloom(4, nb * 10)
        items.append(BatchItem(f, f.alloc_filter_data(), dev(bk), dev(pk),
                               torch.full((len(pk),), -1, dtype=torch.int32, device="cuda"),
                               torch.full((1,), -1, dtype=torch.int64, device="cuda"), 100 * i))
        checks.append((kind, o, bk, pk, 100 * i))
    b = Batch(items, use_graph=False)
    assert b.fallback_count() == 3
    b.run()
    torch.cuda.synchronize()
    for (kind, o, bk, pk, off), it in zip(checks, items):
        words = it.filter_data.cpu().numpy().view(np.uint64)
        if kind != "bcf":
            ref = o.alloc()
            o.insert(ref, bk)
            assert np.array_equal(words, ref), kind
        assert len(o.batch_contains(words, bk)) == len(bk), kind
        exp = o.batch_contains(words, pk, off)
        n = int(it.match_cnt.item())
        assert n == len(exp) and np.array_equal(it.match_positions[:n].cpu().numpy().view(np.uint32), exp), kind
