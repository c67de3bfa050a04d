"""Bit-exact parity with the reference at the benchmark configurations' full sizes.

The reference here is its own filter logic compiled from its sources
(oracle/_ref/libdtlref_*.so: blocked_bloomfilter_logic, cuckoofilter_logic),
run on all host threads.  For every case the WHOLE match list of the GPU's
automatic probe plan is compared with the whole list of the reference's
batch_contains over the same keys (blocked_bloomfilter_batch_dispatch.hpp:
29-69, cuckoofilter_logic.hpp:346-362), and for Bloom filters the GPU-built
words with the words of the reference's own insert:

* the register-blocked filter (u32, w=1, k=4, 16 bits/key, 2^20 build keys,
  2^24 probes at 10 % hits);
* the cache-sectorized filter (u64, w=8, s=8, k=8) at n = 2^22, 2^26 and 2^28
  build keys and 8 / 12 / 16 bits per key, 2^28 probes; at n = 2^28 every hit
  ratio 1 %, 10 % and 50 % (the headline: 16 bits/key, 10 %, the partitioned
  plan over 64 ranges, positions up to 2^28);
* the cuckoo filter (4 tags per bucket, odd MAGIC bucket count) at 2^26 keys,
  16- and 12-bit tags at load 0.95, 8-bit tags at 0.93 (the reference's own
  build of 2^26 keys at 8 bits and 0.95 fails: its victim cache fills), built
  by the reference and probed with 2^28 keys at 10 % hits; and the GPU's own
  build of the same keys, whose false-positive rate on 2^27 non-members must
  equal the reference-built table's within a binomial bound.

Keys are the benchmark's seeded key streams, generated on the device and
copied to the host for the reference.
"""
import os

import numpy as np
import pytest

import dtlg as F
import oracle as O
from dtlg import keygen

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SEED = 20240601   # the benchmark's key seed
THREADS = max(1, len(os.sched_getaffinity(0)))


@pytest.fixture(scope="module")
def ref():
    r = O.try_reflib()
    if r is None:
        pytest.skip("the reference's filter logic (oracle/_ref) is not built")
    return r


def host(t):
    return t.cpu().numpy().view(np.uint32)


def gpu_list(f, words, keys):
    pos = torch.empty(keys.numel(), dtype=torch.int32, device="cuda")
    n = f.batch_contains(words, keys, keys.numel(), pos, 0)
    out = pos[:n].cpu().numpy().view(np.uint32).copy()
    del pos
    return out


def bloom_case(ref, cfg, n, bpk, hits, n_probe):
    wb, w, s, z, k = cfg
    m = n * bpk
    f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                 zone_cnt=z), m)
    rf = ref.bloom(wb, w, s, z, k, m)
    assert rf is not None
    bk = keygen.build_keys_torch(n, SEED)
    words = f.alloc_filter_data()
    assert f.batch_insert(words, bk)
    rw = np.zeros((rf.word_cnt * wb + 7) // 8, dtype=np.uint64)
    rf.insert_mt(rw, host(bk), THREADS)
    del bk
    got = words.cpu().numpy().view(np.uint64)
    assert np.array_equal(got[:len(rw)], rw), "GPU-built words differ from the reference's"
    assert not got[len(rw):].any()
    del got
    out = np.zeros(n_probe + 64, dtype=np.uint32)
    for h in hits:
        keys, member = keygen.probe_keys_torch(n, n_probe, h, SEED)
        want = rf.batch_contains_mt_list(rw, host(keys), THREADS, out=out)
        got = gpu_list(f, words, keys)
        assert len(got) == len(want), (n, bpk, h, len(got), len(want))
        assert np.array_equal(got, want), (n, bpk, h)
        assert len(want) >= int(member.sum().item())
        del keys, member
        torch.cuda.empty_cache()
    del words
    torch.cuda.empty_cache()


def test_register_blocked_baseline_size(ref):
    """u32 w=1 s=1 k=4, m = 16 * 2^20 bits (POW2), 2^20 keys, 2^24 probes."""
    bloom_case(ref, (4, 1, 1, 1, 4), 1 << 20, 16, (0.10,), 1 << 24)


@pytest.mark.parametrize("log2_n", [22, 26])
@pytest.mark.parametrize("bpk", [8, 12, 16])
def test_sectorized_smaller_sizes(ref, log2_n, bpk):
    """L2-resident (2^22 keys, bitmask plan) and just-beyond-L2 (2^26 keys)."""
    bloom_case(ref, (8, 8, 8, 1, 8), 1 << log2_n, bpk, (0.10,), 1 << 28)


@pytest.mark.parametrize("bpk", [16, 8, 12])
def test_sectorized_2p28_every_hit_ratio(ref, bpk):
    """n = 2^28 (256-512 MiB, DRAM-resident, partitioned plan), 2^28 probes."""
    bloom_case(ref, (8, 8, 8, 1, 8), 1 << 28, bpk, (0.10, 0.01, 0.50), 1 << 28)


@pytest.mark.parametrize("t,lf", [(16, 0.95), (12, 0.95), (8, 0.93)])
def test_cuckoo_2p26(ref, t, lf):
    import bench
    n, b = 1 << 26, 4
    m = bench.cuckoo_bits(n, t, b, lf)
    f = F.cf(m, t, b)
    rf = ref.cuckoo(t, b, m)
    assert rf is not None and f.block_cnt() % 2 == 1 and f.is_magic()
    bk = keygen.build_keys_torch(n, SEED)
    # the reference's build (single thread: its inserts are not thread-safe).
    # Its kicks draw from a random generator it seeds itself, so at load 0.95
    # an attempt now and then ends with a key it cannot place; another attempt
    # (the generator moves on) is a new random build of the same keys.
    for attempt in range(3):
        table = np.zeros(f.alloc_words(), dtype=np.uint64)
        assert (rf.word_cnt * 4 + 12) <= table.nbytes
        if rf.insert(table, host(bk)):
            break
    else:
        raise AssertionError("the reference's build lost keys in 3 attempts")
    assert rf.count_occupied(table) == n
    # the GPU's probe of the reference-built table == the reference's probe
    words = torch.from_numpy(table.view(np.int64)).cuda()
    out = np.zeros((1 << 28) + 64, dtype=np.uint32)
    keys, member = keygen.probe_keys_torch(n, 1 << 28, 0.10, SEED)
    want = rf.batch_contains_mt_list(table, host(keys), THREADS, out=out)
    got = gpu_list(f, words, keys)
    assert np.array_equal(got, want), (t, len(got), len(want))
    assert len(want) >= int(member.sum().item())
    del keys, member, words
    # the GPU's build of the same keys: all placed, same false-positive rate
    gw = f.alloc_filter_data()
    assert f.batch_insert(gw, bk), f"GPU build lost {f.last_failed} keys"
    assert f.count_occupied_slots(gw) == n
    assert len(gpu_list(f, gw, bk)) == n          # no false negatives
    neg, _ = keygen.probe_keys_torch(n, 1 << 27, 0.0, SEED + 1)
    fp_gpu = len(gpu_list(f, gw, neg))
    fp_ref = len(rf.batch_contains_mt_list(table, host(neg), THREADS, out=out))
    # both tables hold the same tags in differently chosen buckets: equal
    # rates, counts within 5 standard deviations of their difference
    assert abs(fp_gpu - fp_ref) <= 5 * np.sqrt(fp_gpu + fp_ref) + 5, (t, fp_gpu, fp_ref)
    del gw, neg, bk
    torch.cuda.empty_cache()
