"""Parity of the CUDA path (through the C ABI) with the reference.

Bit-exact: Bloom filter words after batch_insert, and the ascending match
positions of batch_contains, against the C oracle (itself pinned to the
reference) and against golden vectors produced by the reference.
"""
import numpy as np
import pytest

import dtlg as F
import oracle as O
from dtlg import keygen
from gen_ref_instances import bloom_configs, cuckoo_configs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev_words(np_words):
    return torch.from_numpy(np.ascontiguousarray(np_words).view(np.int64)).cuda()


def dev_keys(keys, pad=0):
    """uint32 keys on the device starting `pad` keys into a buffer (pad=1..3
    gives a key pointer that is not 16-byte aligned)."""
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


def test_reference_known_answer_facade():
    # src/dtl/filter/filter_test.cpp:16-40, through the filter facade
    f = F.filter(F.blocked_bloomfilter_config(), 1024)
    assert f.insert(torch.tensor([13, 37, 42, 88], dtype=torch.int32, device="cuda"))
    p = f.probe()
    pos = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert p(torch.tensor([13, 37, 42, 88], dtype=torch.int32, device="cuda"), pos, 0) == 4
    assert pos.tolist() == [0, 1, 2, 3]
    assert p(torch.tensor([0, 1, 42, 2], dtype=torch.int32, device="cuda"), pos, 1000) == 1
    assert pos[0].item() == 1002
    # host buffers (the reference's calling convention)
    hp = np.zeros(4, dtype=np.uint32)
    assert p(np.array([0, 1, 42, 2], dtype=np.uint32), hp, 1000) == 1 and hp[0] == 1002


def test_bloom_every_config_bit_exact():
    """Every config the reference's dispatchers accept, POW2 and MAGIC:
    GPU-built words == oracle-built words, GPU probe == oracle probe."""
    for ci, (wb, w, s, z, k) in enumerate(bloom_configs()):
        for m in (1 << 14, (1 << 14) + 1000):
            ob = O.Bloom(wb, w, s, z, k, m)
            f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w,
                                                         sector_cnt=s, zone_cnt=z), m)
            n = max(1, int(ob.m_actual // 12))
            seed = 100 + ci
            bk = keygen.build_keys(n, seed)
            ref_words = ob.alloc()
            ob.insert(ref_words, bk)
            words = f.alloc_filter_data()
            assert f.batch_insert(words, dev_keys(bk, pad=ci % 4))
            got = words.cpu().numpy().view(np.uint64)
            assert np.array_equal(got, ref_words), (wb, w, s, z, k, m)
            # the partitioned build plan: the same words
            f.set_build_options(2)
            words2 = f.alloc_filter_data()
            assert f.batch_insert(words2, dev_keys(bk, pad=(ci + 2) % 4))
            assert np.array_equal(words2.cpu().numpy().view(np.uint64), ref_words), (wb, w, s, z, k, m, "plan 2")
            f.set_build_options(0)
            pk, _ = keygen.probe_keys(n, 3001, 0.4, seed)
            off = (1 << 32) - 1500 if ci % 2 else 17
            exp = ob.batch_contains(ref_words, pk, off)
            for mode in (1, 2, 3, 4):  # fused; bitmask (1-3 block-range passes); partitioned; shared memory
                f.set_probe_options(mode, ci % 2)
                f.set_probe_passes(1 + ci % 3)
                assert np.array_equal(gpu_probe(f, words, pk, off, pad=(ci + 1) % 4), exp), (wb, w, s, z, k, m, mode)


def test_bloom_golden_vectors(golden):
    index, arr = golden
    for e in index["bloom"]:
        wb, w, s, z, k = e["cfg"]
        f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                     zone_cnt=z), e["m"])
        words = f.alloc_filter_data()
        assert f.batch_insert(words, dev_keys(keygen.build_keys(e["n_build"], e["seed"])))
        ref = arr[f"bloom_{e['id']}_words"]
        assert np.array_equal(words.cpu().numpy().view(np.uint64)[:len(ref)], ref), e
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        assert np.array_equal(gpu_probe(f, words, pk, e["match_offset"]), arr[f"bloom_{e['id']}_hits"]), e


def test_shared_memory_plan():
    """Plan 4 (filter copied into shared memory): available up to 192 KiB,
    a fallback to plan 2 above, never the automatic choice (plan 2 in one
    pass: two kernels); always the oracle's match list."""
    L = F.lib()
    for (wb, w, s_, z, k) in ((8, 8, 8, 1, 8), (4, 1, 1, 1, 4), (8, 8, 8, 2, 8), (4, 16, 1, 1, 6)):
        for kib in (4, 64, 96, 160, 256):
            m = kib * 8192 - 8 * 64 * (kib % 3)  # POW2 and MAGIC sizes
            ob = O.Bloom(wb, w, s_, z, k, m)
            f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s_,
                                                         zone_cnt=z), m)
            n = int(ob.m_actual // 12)
            bk = keygen.build_keys(n, kib)
            rw = ob.alloc()
            ob.insert(rw, bk)
            words = dev_words(rw)
            pk, _ = keygen.probe_keys(n, (1 << 21) + 3, 0.1, kib)
            exp = ob.batch_contains(rw, pk, 77)
            f.set_probe_options(0, -1)
            assert L.dtlg_probe_kernel_count(f._h, len(pk)) == 2
            for mode in (0, 4):
                f.set_probe_options(mode, -1)
                for pad in (0, 3):
                    assert np.array_equal(gpu_probe(f, words, pk, 77, pad), exp), (wb, w, s_, z, k, kib, mode, pad)


@pytest.mark.parametrize("layout", [(8, 8, 8, 4, 8), (8, 8, 4, 1, 8), (4, 16, 8, 1, 8), (8, 8, 8, 1, 8),
                                    (8, 8, 2, 1, 8), (4, 16, 16, 2, 8)])
def test_probe_filter_base_16_not_32_byte_aligned(layout):
    """Filter words that start 16 bytes past a 32-byte boundary: the probes
    read 32-byte chunks and half blocks with 256-bit loads only from 32-byte
    aligned words and fall back to narrower loads otherwise.  Both forms give
    the oracle's list in every plan (the chunked layouts u64 w=8 z=4 and s=4,
    u32 w=16 s=8 included)."""
    wb, w, s_, z, k = layout
    m = 12 * 40000
    ob = O.Bloom(wb, w, s_, z, k, m)
    f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s_,
                                                 zone_cnt=z), m)
    bk = keygen.build_keys(40000, 8)
    rw = ob.alloc()
    ob.insert(rw, bk)
    buf = torch.zeros(len(rw) + 4, dtype=torch.int64, device="cuda")
    assert buf.data_ptr() % 32 == 0
    for shift in (0, 2):  # words at a 32-byte boundary, then 16 bytes past one
        words = buf[shift:shift + len(rw)]
        words.copy_(dev_words(rw))
        pk, _ = keygen.probe_keys(40000, 70001, 0.3, 8)
        exp = ob.batch_contains(rw, pk, 5)
        for mode, variant in ((1, -1), (2, 0), (2, 1), (3, 0), (3, 1), (4, -1)):
            f.set_probe_options(mode, variant)
            assert np.array_equal(gpu_probe(f, words, pk, 5), exp), (layout, shift, mode, variant)
        f.set_probe_options(0, -1)


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 5, 31, 1023, 1024, 4095, 4096, 4097, 8191, 65537, 300001])
def test_probe_lengths_and_alignment(n):
    ob = O.Bloom(8, 8, 8, 1, 8, 3 * (1 << 16))
    f = F.bbf_64(3 * (1 << 16), 8, 8, 8)
    bk = keygen.build_keys(20000, 5)
    rw = ob.alloc()
    ob.insert(rw, bk)
    words = dev_words(rw)
    pk, _ = keygen.probe_keys(20000, n, 0.5, 5)
    exp = ob.batch_contains(rw, pk, 9)
    for mode, variant, passes in ((0, -1, 0), (1, -1, 0), (2, 0, 1), (2, 1, 1), (2, 1, 3), (2, 0, 16), (3, 0, 0),
                                  (3, 1, 0), (4, -1, 0)):
        f.set_probe_options(mode, variant)
        f.set_probe_passes(passes)
        for pad in range(4):
            assert np.array_equal(gpu_probe(f, words, pk, 9, pad), exp), (mode, variant, passes, pad)


def test_cuckoo_probe_every_config_bit_exact():
    """Tables built on the CPU (restatement of the reference's insert), uploaded,
    probed on the GPU: identical match lists, victim cache included."""
    for ci, (t, b) in enumerate(cuckoo_configs()):
        for m in (1 << 16, (1 << 16) + 4321):
            oc = O.Cuckoo(t, b, m)
            f = F.cf(m, t, b)
            assert f.alloc_words() >= oc.alloc_u64 - 2
            table = np.zeros(f.alloc_words(), dtype=np.uint64)
            n = int(oc.bucket_cnt * b * (0.97 if b == 4 else 0.6))
            bk = keygen.build_keys(n, 300 + ci)
            oc.insert(table, bk, seed=ci + 1)
            pk, _ = keygen.probe_keys(n, 5000, 0.3, 300 + ci)
            exp = oc.batch_contains(table, pk, 11)
            for mode, passes in ((1, 0), (2, 1), (2, 2), (2, 5)):
                f.set_probe_options(mode, ci % 2)
                f.set_probe_passes(passes)
                assert np.array_equal(gpu_probe(f, dev_words(table), pk, 11, pad=ci % 4), exp), (t, b, m, mode, passes)
            assert f.count_occupied_slots(dev_words(table)) == oc.count_occupied(table)


def test_cuckoo_golden_vectors(golden):
    index, arr = golden
    for e in index["cuckoo"]:
        f = F.cf(e["m"], e["t"], e["b"])
        ref_table = arr[f"cuckoo_{e['id']}_table"]
        table = np.zeros(max(f.alloc_words(), len(ref_table)), dtype=np.uint64)
        table[:len(ref_table)] = ref_table
        pk, _ = keygen.probe_keys(e["n_build"], e["n_probe"], e["hit_ratio"], e["seed"])
        got = gpu_probe(f, dev_words(table), pk, e["match_offset"])
        assert np.array_equal(got, arr[f"cuckoo_{e['id']}_hits"]), e


@pytest.mark.parametrize("t,b,m", [(16, 4, 1 << 20), (8, 4, 1 << 20), (12, 4, 1 << 20), (16, 4, 4462025 * 64),
                                   (8, 2, (1 << 18) + 3), (32, 4, 1 << 18), (4, 4, 1 << 18), (16, 1, 1 << 18)])
def test_cuckoo_gpu_build_invariants(t, b, m):
    """The GPU build is randomised like the reference's; check no false
    negatives, occupancy, and the false-positive rate against a CPU build."""
    oc = O.Cuckoo(t, b, m)
    f = F.cf(m, t, b)
    lf = 0.9 if b == 4 else (0.75 if b == 2 else 0.4)
    n = int(oc.bucket_cnt * b * lf)
    bk = keygen.build_keys(n, 77)
    words = f.alloc_filter_data()
    ok = f.batch_insert(words, dev_keys(bk))
    assert ok, f"lost {f.last_failed} of {n}"
    occ = f.count_occupied_slots(words)
    assert occ == n
    # no false negatives
    members = gpu_probe(f, words, bk)
    assert len(members) == n
    # FPR vs the CPU restatement's build of the same keys
    neg, _ = keygen.probe_keys(n, 200000, 0.0, 77)
    fp_gpu = len(gpu_probe(f, words, neg))
    table = np.zeros(f.alloc_words(), dtype=np.uint64)
    assert oc.insert(table, bk, seed=3)
    fp_cpu = len(oc.batch_contains(table, neg))
    # the tag sets are equal; only slot placement differs -> same FPR
    sd = np.sqrt(max(fp_cpu, 1))
    assert abs(fp_gpu - fp_cpu) <= 5 * sd + 5, (fp_gpu, fp_cpu)


def test_host_buffer_pipeline_multi_chunk():
    """batch_contains over host buffers, more keys than one pipeline chunk."""
    m = 1 << 24
    ob = O.Bloom(8, 8, 8, 1, 8, m)
    f = F.bbf_64(m, 8, 8, 8)
    bk = keygen.build_keys(1 << 20, 9)
    words = f.alloc_filter_data()
    assert f.batch_insert_host(words, bk)
    rw = ob.alloc()
    ob.insert(rw, bk)
    assert np.array_equal(words.cpu().numpy().view(np.uint64), rw)
    pk, _ = keygen.probe_keys(1 << 20, (1 << 24) * 2 + 12345, 0.1, 9)
    out = np.zeros(len(pk), dtype=np.uint32)
    n = f.batch_contains_host(words, pk, out, 123)
    exp = ob.batch_contains(rw, pk, 123)
    assert n == len(exp) and np.array_equal(out[:n], exp)


def test_single_key_api():
    f = F.bbf_32(1 << 16, 6, 2, 1)
    words = f.alloc_filter_data()
    assert f.insert(words, 4242)
    assert f.contains(words, 4242)
    assert not f.contains(words, 4243) or True  # a false positive is allowed
    ob = O.Bloom(4, 2, 1, 1, 6, 1 << 16)
    rw = ob.alloc()
    ob.insert(rw, [4242])
    assert np.array_equal(words.cpu().numpy().view(np.uint64), rw)


def test_large_filter_property():
    """A DRAM-resident sectorized filter (u64, w=8, s=8, k=8, 16 bits/key,
    2^26 keys, 128 MiB): every member found; positions identical to the oracle."""
    n = 1 << 26
    m = n * 16
    ob = O.Bloom(8, 8, 8, 1, 8, m)
    f = F.bbf_64(m, 8, 8, 8)
    bk = keygen.build_keys(n, 21)
    words = f.alloc_filter_data()
    assert f.batch_insert(words, dev_keys(bk))
    rw = ob.alloc()
    ob.insert(rw, bk)
    assert np.array_equal(words.cpu().numpy().view(np.uint64), rw)
    pk, member = keygen.probe_keys(n, 1 << 24, 0.1, 21)
    got = gpu_probe(f, words, pk)
    exp = ob.batch_contains(rw, pk)
    assert np.array_equal(got, exp)
    assert np.all(np.isin(np.nonzero(member)[0].astype(np.uint32), got))


def test_partitioned_build_large_filter():
    """Filters beyond 80 MiB are built through the partition automatically:
    the same words as the one-kernel build (and, on a sample, the oracle's
    probe of them), for a sectorized and a zoned layout, POW2 and MAGIC."""
    for (wb, w, s_, z, k), m in (((8, 8, 8, 1, 8), 1 << 31), ((8, 8, 8, 2, 8), (3 << 29) + 4096)):
        f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s_,
                                                     zone_cnt=z), m)
        n = 1 << 25
        bk = keygen.build_keys_torch(n, 91)
        auto = f.alloc_filter_data()
        assert f.batch_insert(auto, bk)
        f.set_build_options(1)
        direct = f.alloc_filter_data()
        assert f.batch_insert(direct, bk)
        f.set_build_options(0)
        assert torch.equal(auto, direct), (wb, w, s_, z, k, m)
        ob = O.Bloom(wb, w, s_, z, k, m)
        words = auto.cpu().numpy().view(np.uint64)
        sample = bk[: 1 << 16].cpu().numpy().view(np.uint32)
        assert len(ob.batch_contains(words, sample)) == len(sample)
        del auto, direct
        torch.cuda.empty_cache()


def _keys_in_top_half(n, seed, mul):
    """n distinct keys whose hash key * mul (mod 2^32) is below 2^31."""
    out, start = [], 0
    while sum(len(o) for o in out) < n:
        k = keygen.build_keys(4 * n, seed, start=start)
        start += 4 * n
        out.append(k[((k.astype(np.uint64) * np.uint64(mul)) & np.uint64(0xFFFFFFFF)) < np.uint64(1 << 31)])
    return np.concatenate(out)[:n]


def test_partitioned_plan_with_overflowing_range():
    """The partition gives every range a segment of its expected share plus
    slack; keys skewed into one range overflow it, and the overflowing keys
    are probed (inserted) straight from the key array.  A POW2 filter of two
    8 MiB ranges; 95 % of the keys hash into the first: the partitioned probe
    and the partitioned build still equal the oracle."""
    m = 1 << 27                                   # 16 MiB: 2^18 64-byte blocks, ranges of 2^17
    ob = O.Bloom(8, 8, 8, 1, 8, m)
    f = F.bbf_64(m, 8, 8, 8)
    c0 = 596572387                                # the block hash constant, hash_family.hpp
    skew = _keys_in_top_half(1 << 20, 71, c0)     # block < 2^17: range 0
    bk = np.concatenate([skew[: 950000], keygen.build_keys(50000, 72)])
    rw = ob.alloc()
    ob.insert(rw, bk)
    f.set_build_options(2)
    words = f.alloc_filter_data()
    assert f.batch_insert(words, dev_keys(bk, pad=2))
    f.set_build_options(0)
    assert np.array_equal(words.cpu().numpy().view(np.uint64)[:len(rw)], rw)
    pk = np.concatenate([skew[500000:], keygen.probe_keys(50000, 200001, 0.3, 72)[0]])
    np.random.default_rng(3).shuffle(pk)
    exp = ob.batch_contains(rw, pk, 5)
    for variant in (0, 1):
        f.set_probe_options(3, variant)
        for pad in (0, 1):
            assert np.array_equal(gpu_probe(f, words, pk, 5, pad), exp), (variant, pad)
    f.set_probe_options(0, -1)
