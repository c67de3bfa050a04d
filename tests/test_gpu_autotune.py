"""The autotuners pick a probe plan / batch launch shape by timing; whatever
they pick, results stay bit-exact."""
import numpy as np
import pytest

import dtlg as F
import oracle as O
from dtlg import keygen

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("cfg,m", [((8, 8, 8, 1, 8), 1 << 26), ((4, 16, 16, 2, 8), (1 << 29) + 4096),
                                   ((4, 1, 1, 1, 4), 1 << 24)])
def test_probe_autotune_keeps_results(cfg, m):
    wb, w, s, z, k = cfg
    f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                 zone_cnt=z), m)
    n = m // 16
    ob = O.Bloom(wb, w, s, z, k, m)
    bk = keygen.build_keys(n, 31)
    pk, _ = keygen.probe_keys(n, 1 << 21, 0.1, 31)
    rw = ob.alloc()
    ob.insert(rw, bk)
    exp = ob.batch_contains(rw, pk, 9)
    data = torch.from_numpy(rw.view(np.int64)).cuda()
    keys = torch.from_numpy(pk.view(np.int32)).cuda()
    plan = f.autotune(data, keys, reps=3)
    assert plan["mode"] in (1, 2, 3) and plan["ms"] > 0 and plan["gkeys_per_s"] > 0
    pos = torch.empty(len(pk), dtype=torch.int32, device="cuda")
    c = f.batch_contains(data, keys, len(pk), pos, 9)
    assert c == len(exp)
    assert np.array_equal(pos[:c].cpu().numpy().view(np.uint32), exp)


def test_cuckoo_probe_autotune_keeps_results():
    m = 1 << 24
    ob = O.Cuckoo(16, 4, m)
    f = F.cf(m, 16, 4)
    rw = ob.alloc()
    bk = keygen.build_keys(int(ob.bucket_cnt * 4 * 0.7), 5)
    assert ob.insert(rw, bk)
    pk, _ = keygen.probe_keys(len(bk), 1 << 20, 0.1, 5)
    exp = ob.batch_contains(rw, pk, 0)
    data = torch.from_numpy(rw.view(np.int64)).cuda()
    keys = torch.from_numpy(pk.view(np.int32)).cuda()
    f.autotune(data, keys, reps=2)
    pos = torch.empty(len(pk), dtype=torch.int32, device="cuda")
    c = f.batch_contains(data, keys, len(pk), pos, 0)
    assert np.array_equal(pos[:c].cpu().numpy().view(np.uint32), exp)


def test_batch_autotune_keeps_results():
    from dtlg.batch import Batch, BatchItem
    items, refs = [], []
    for i, (cfg, n) in enumerate([((8, 8, 8, 4, 8), 300000), ((4, 16, 16, 2, 8), 50000), ((4, 1, 1, 1, 8), 2000)]):
        wb, w, s, z, k = cfg
        m = n * 12 + 100
        f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                     zone_cnt=z), m)
        ob = O.Bloom(wb, w, s, z, k, m)
        bk = keygen.build_keys(n, 60 + i)
        pk, _ = keygen.probe_keys(n, 3 * n, 0.05, 60 + i)
        rw = ob.alloc()
        ob.insert(rw, bk)
        refs.append((rw, ob.batch_contains(rw, pk, 0)))
        items.append(BatchItem(f, f.alloc_filter_data(), torch.from_numpy(bk.view(np.int32)).cuda(),
                               torch.from_numpy(pk.view(np.int32)).cuda(),
                               torch.zeros(len(pk), dtype=torch.int32, device="cuda"),
                               torch.zeros(1, dtype=torch.int64, device="cuda"), 0))
    b = Batch(items)
    plan = b.autotune(reps=2)
    assert plan["staging"] in (0, 1) and plan["ms"] > 0
    for it in items:
        it.filter_data.zero_()
    b.run()
    torch.cuda.synchronize()
    for (rw, exp), it in zip(refs, items):
        assert np.array_equal(it.filter_data.cpu().numpy().view(np.uint64), rw)
        c = int(it.match_cnt.item())
        assert np.array_equal(it.match_positions[:c].cpu().numpy().view(np.uint32), exp)
