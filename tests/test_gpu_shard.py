"""dtlg_or_words, the device OR of sharded Bloom builds, against numpy; and a
sharded build on one GPU (world size 1 of the same code) against the full one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

import dtlg as F  # noqa: E402
from dtlg import keygen  # noqa: E402
from dtlg.shard import or_words, shard_bounds  # noqa: E402


@pytest.mark.parametrize("n,parts", [(1, 1), (1000003, 3), (1 << 22, 4)])
def test_or_words_matches_numpy(n, parts):
    rng = np.random.default_rng(n)
    dst = rng.integers(0, 2 ** 63, n, dtype=np.int64)
    src = [rng.integers(0, 2 ** 63, n, dtype=np.int64) for _ in range(parts)]
    d = torch.from_numpy(dst.copy()).cuda()
    or_words(d, [torch.from_numpy(s).cuda() for s in src])
    want = dst.copy()
    for s in src:
        want |= s
    assert np.array_equal(d.cpu().numpy(), want)


def test_partial_builds_or_to_the_full_build():
    cfg = F.blocked_bloomfilter_config(k=8, word_size=8, word_cnt_per_block=8, sector_cnt=8)
    n, world = 1 << 20, 4
    f = F.construct(cfg, n * 12 + 5)
    keys = keygen.build_keys_torch(n, 9)
    parts = []
    for r in range(world):
        a, c = shard_bounds(n, r, world)
        w = f.alloc_filter_data()
        assert f.batch_insert(w, keys[a:a + c].contiguous())
        parts.append(w)
    full = f.alloc_filter_data()
    assert f.batch_insert(full, keys)
    combined = parts[0].clone()
    or_words(combined, parts[1:])
    assert torch.equal(combined, full)


def test_facade_replica_path_returns_the_oracles_list():
    """filter.probe() probes the replica of the keys' device.  On one GPU the
    home words are that replica; the copy a second device would get
    (dtlg_copy_words_peer, here device 0 -> device 0) is bit-identical and
    probes to the same list, the oracle's."""
    import importlib

    import numpy as np
    import oracle as O
    from dtlg import keygen
    Fm = importlib.import_module("dtlg.filter")
    m = 12 * 100000 + 77
    f = F.filter(F.blocked_bloomfilter_config(k=8, word_size=8, word_cnt_per_block=8, sector_cnt=8), m)
    bk = keygen.build_keys(100000, 61)
    assert f.insert(torch.from_numpy(bk.view(np.int32)).cuda())
    ob = O.Bloom(8, 8, 8, 1, 8, m)
    rw = ob.alloc()
    ob.insert(rw, bk)
    pk, _ = keygen.probe_keys(100000, 300000, 0.2, 61)
    want = ob.batch_contains(rw, pk, 3)
    keys = torch.from_numpy(pk.view(np.int32)).cuda()
    p = f.probe()
    out = torch.zeros(len(pk), dtype=torch.int32, device="cuda")
    n = p(keys, out, 3)
    assert np.array_equal(out[:n].cpu().numpy().view(np.uint32), want)
    assert f.replicas.devices() == [0]                       # no copy for the home device
    copy = Fm._peer_replica(f.filter_data, 0)
    assert copy.data_ptr() != f.filter_data.data_ptr() and torch.equal(copy, f.filter_data)
    out2 = torch.zeros(len(pk), dtype=torch.int32, device="cuda")
    n2 = f.filter_instance.batch_contains(copy, keys, len(pk), out2, 3)
    assert n2 == n and torch.equal(out2[:n2], out[:n])
    # host keys go to the current device's replica
    hp = np.zeros(len(pk), dtype=np.uint32)
    assert p(pk, hp, 3) == n and np.array_equal(hp[:n], want)
    if torch.cuda.device_count() > 1:
        k1 = keys.to("cuda:1")
        o1 = torch.zeros(len(pk), dtype=torch.int32, device="cuda:1")
        assert p(k1, o1, 3) == n and np.array_equal(o1[:n].cpu().numpy().view(np.uint32), want)
        assert f.replicas.devices() == [0, 1]
