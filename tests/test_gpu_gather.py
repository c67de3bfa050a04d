"""Probe -> gather: the matching rows of payload columns, in match order,
against numpy indexing by the oracle's match list."""
import numpy as np
import pytest

import dtlg as F
import oracle as O
from dtlg import keygen

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def build(cfg, m, n, seed):
    wb, w, s, z, k = cfg
    f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                 zone_cnt=z), m)
    ob = O.Bloom(wb, w, s, z, k, m)
    rw = ob.alloc()
    ob.insert(rw, keygen.build_keys(n, seed))
    return f, ob, rw


@pytest.mark.parametrize("mode", [0, 2, 3])
@pytest.mark.parametrize("n_probe,pre", [(1, 0), (4097, 1), (300001, 3)])
def test_gather_matches_numpy(mode, n_probe, pre):
    cfg, n = (8, 8, 8, 1, 8), 100000
    f, ob, rw = build(cfg, n * 12 + 9, n, 3)
    f.set_probe_options(mode, -1)
    pk, _ = keygen.probe_keys(n, n_probe, 0.3, 3)
    exp = ob.batch_contains(rw, pk, 17)
    data = torch.from_numpy(rw.view(np.int64)).cuda()
    store = torch.from_numpy(np.concatenate([np.zeros(pre, np.uint32), pk]).view(np.int32)).cuda()
    keys = store[pre:]                                   # misaligned by `pre` keys
    rng = np.random.default_rng(n_probe)
    c32 = rng.integers(0, 2 ** 31, n_probe, dtype=np.int32)
    c64 = rng.integers(0, 2 ** 62, n_probe, dtype=np.int64)
    cols = [torch.from_numpy(c32).cuda(), torch.from_numpy(c64).cuda()]
    outs = [torch.full((n_probe,), -1, dtype=torch.int32, device="cuda"),
            torch.full((n_probe,), -1, dtype=torch.int64, device="cuda")]
    pos = torch.full((n_probe,), -1, dtype=torch.int32, device="cuda")
    cnt = f.batch_contains_gather(data, keys, cols, outs, pos, 17)
    assert cnt == len(exp)
    assert np.array_equal(pos[:cnt].cpu().numpy().view(np.uint32), exp)
    idx = exp.astype(np.int64) - 17
    assert np.array_equal(outs[0][:cnt].cpu().numpy(), c32[idx])
    assert np.array_equal(outs[1][:cnt].cpu().numpy(), c64[idx])
    # positions are optional when payload is gathered
    outs2 = [torch.zeros(n_probe, dtype=torch.int64, device="cuda")]
    assert f.batch_contains_gather(data, keys, cols[1:], outs2) == cnt
    assert np.array_equal(outs2[0][:cnt].cpu().numpy(), c64[idx])


def test_gather_cuckoo():
    m = 1 << 22
    ob = O.Cuckoo(16, 4, m)
    f = F.cf(m, 16, 4)
    rw = ob.alloc()
    bk = keygen.build_keys(int(ob.bucket_cnt * 4 * 0.7), 8)
    assert ob.insert(rw, bk)
    pk, _ = keygen.probe_keys(len(bk), 200000, 0.2, 8)
    exp = ob.batch_contains(rw, pk, 0)
    data = torch.from_numpy(rw.view(np.int64)).cuda()
    col = torch.arange(len(pk), dtype=torch.int32, device="cuda") * 3
    out = torch.zeros(len(pk), dtype=torch.int32, device="cuda")
    cnt = f.batch_contains_gather(data, torch.from_numpy(pk.view(np.int32)).cuda(), [col], [out])
    assert cnt == len(exp)
    assert np.array_equal(out[:cnt].cpu().numpy(), exp.astype(np.int64) * 3)
