"""Full-size properties (the benchmark sizes, beyond what the oracle checks in
seconds): no false negatives, strictly ascending positions, identical lists
from every probe plan, and a false-positive rate at the analytic value."""
import numpy as np
import pytest

import dtlg as F
from dtlg import keygen
from dtlg.model.candidates import Candidate

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def probe(f, words, keys, offset=0, mode=0, passes=0):
    f.set_probe_options(mode, -1)
    f.set_probe_passes(passes)
    pos = torch.empty(keys.numel(), dtype=torch.int32, device="cuda")
    n = f.batch_contains(words, keys, keys.numel(), pos, offset)
    f.set_probe_options(0, -1)
    f.set_probe_passes(0)
    return n, pos


@pytest.mark.parametrize("log2_n,bpk,sizing", [(28, 12, "exact"), (28, 12, "uncorrelated"), (26, 16, "exact")])
def test_sectorized_full_size(log2_n, bpk, sizing):
    """`exact`: m = n * bits per key, as the benchmark configurations size it
    (2^28 x 12 bits gives 3 * 2^21 MAGIC blocks, whose FPR the reference's
    hashing inflates: checked against the reference's behaviour elsewhere, not
    the analytic value); `uncorrelated`: the planner's sizing."""
    from dtlg.model.planner import uncorrelated_bits
    n = 1 << log2_n
    cand = Candidate("bloom", 8, 8, 8, 1, 8)
    m = n * bpk if sizing == "exact" else uncorrelated_bits(cand, n * bpk)
    f = F.construct(F.blocked_bloomfilter_config(k=8, word_size=8, word_cnt_per_block=8, sector_cnt=8), m)
    words = f.alloc_filter_data()
    assert f.batch_insert(words, keygen.build_keys_torch(n, 41))
    # every build key is found: the list is exactly 0 .. n-1
    members = keygen.build_keys_torch(n, 41)
    cnt, pos = probe(f, words, members)
    assert cnt == n
    assert torch.equal(pos[:n], torch.arange(n, dtype=torch.int32, device="cuda"))
    del members, pos
    # half members, half non-members: every plan gives the same ascending list
    keys, member = keygen.probe_keys_torch(n, 1 << 26, 0.5, 41)
    lists = []
    for mode, passes in ((0, 0), (2, 1), (2, 3), (3, 0)):
        c, p = probe(f, words, keys, 7, mode, passes)
        lists.append(p[:c].clone())
        del p
    for other in lists[1:]:
        assert torch.equal(lists[0], other)
    got = lists[0].to(torch.int64) - 7
    assert bool((got[1:] > got[:-1]).all())
    hits = torch.zeros(keys.numel(), dtype=torch.bool, device="cuda")
    hits[got] = True
    assert bool(hits[member].all())                          # no false negatives
    fp = int((hits & ~member).sum().item()) / int((~member).sum().item())
    analytic = float(cand.fpr(f.size_in_bytes() * 8 / n))
    if sizing == "uncorrelated":
        assert abs(fp / analytic - 1.0) < 0.1, (fp, analytic)
    elif not f.is_magic():
        # POW2 blocks come from the top bits of the same multiplicative hash
        # family; at 2^26 - 2^28 keys the measured rate is 0.6 - 1.15 x analytic
        assert 0.5 < fp / analytic < 1.5, (fp, analytic)
    else:
        assert fp > analytic  # the correlated MAGIC sizing (see uncorrelated_bits)


def test_cuckoo_full_size():
    import bench
    n = 1 << 26
    m = bench.cuckoo_bits(n, 16, 4, 0.95)
    f = F.cf(m, 16, 4)
    words = f.alloc_filter_data()
    assert f.batch_insert(words, keygen.build_keys_torch(n, 43))
    assert f.count_occupied_slots(words) == n
    members = keygen.build_keys_torch(n, 43)
    cnt, pos = probe(f, words, members)
    assert cnt == n and torch.equal(pos[:n], torch.arange(n, dtype=torch.int32, device="cuda"))
    del members, pos
    keys, member = keygen.probe_keys_torch(n, 1 << 27, 0.0, 43)
    cnt, pos = probe(f, words, keys)
    fp = cnt / keys.numel()
    lf = n / (f.block_cnt() * 4)
    analytic = float(Candidate("cuckoo", t=16, b=4).fpr(16 / lf))
    # The reference's cuckoo FPR formula (math.hpp:198-205) is an estimate that
    # these keys undercut (measured 0.50 x at 2^26 keys, load 0.95); the equality
    # of GPU-built and CPU-built FPR is checked in test_gpu_parity.
    assert 0.25 < fp / analytic < 1.1, (fp, analytic)
