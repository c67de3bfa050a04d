"""The C ABI on the host only (no GPU): the library loads, exports every entry
point include/dtlg.h declares, and constructs / sizes / names filters exactly
as the reference (checked against the C oracle and the golden vectors)."""
import os
import re

import pytest

import oracle as O
from dtlg import _lib
import dtlg as F
from gen_ref_instances import bloom_configs, cuckoo_configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            src = open(os.path.join(inc, fn)).read()
            names |= set(re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(dtlg_\w+)\s*\(", src, re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    decl = declared_functions()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert set(_lib.SIGNATURES) <= decl


def test_version():
    assert b"sm_100a" in _lib.lib().dtlg_version()


@pytest.mark.parametrize("m", [1 << 14, (1 << 14) + 1000, 999, 1, 0, 1 << 33, 3 << 30])
def test_bloom_sizes_match_oracle(m):
    for (wb, w, s, z, k) in bloom_configs():
        cfg = F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s, zone_cnt=z)
        try:
            ob = O.Bloom(wb, w, s, z, k, m)
        except ValueError:
            with pytest.raises(_lib.DtlgError):
                F.construct(cfg, m)
            continue
        f = F.construct(cfg, m)
        assert f.size() == ob.size_u64
        assert f.alloc_words() == ob.size_u64
        assert f.size_in_bytes() == (ob.m_actual + 7) // 8
        assert f.block_cnt() == ob.block_cnt
        assert f.is_magic() == ob.magic


@pytest.mark.parametrize("m", [1 << 16, (1 << 16) + 12345, 5000, 0, 1 << 40])
def test_cuckoo_sizes_match_oracle(m):
    for (t, b) in cuckoo_configs():
        try:
            oc = O.Cuckoo(t, b, m)
        except ValueError:
            with pytest.raises(_lib.DtlgError):
                F.cf(m, t, b)
            continue
        f = F.cf(m, t, b)
        assert f.size() == oc.size_u64
        assert f.alloc_words() >= oc.alloc_u64 - 2
        assert f.alloc_words() * 8 >= oc.table_words_u32 * 4 + 12 + 16
        assert f.block_cnt() == oc.bucket_cnt


def test_invalid_configs_raise_like_reference():
    # blocked_bloomfilter.hpp:106-115 (invalid_argument), filter.hpp:64 (runtime_error)
    bad = [dict(k=3, word_size=4, word_cnt_per_block=1, sector_cnt=2),
           dict(k=8, word_size=4, word_cnt_per_block=1, sector_cnt=8),   # s > w * word bytes
           dict(k=17, word_size=8, word_cnt_per_block=8, sector_cnt=8),
           dict(k=8, word_size=4, word_cnt_per_block=3, sector_cnt=1),
           dict(k=8, word_size=8, word_cnt_per_block=4, sector_cnt=4, zone_cnt=4),  # w <= z
           dict(k=7, word_size=8, word_cnt_per_block=8, sector_cnt=8, zone_cnt=2)]
    for kw in bad:
        with pytest.raises(_lib.InvalidConfig):
            F.construct(F.blocked_bloomfilter_config(**kw), 1 << 16)
    with pytest.raises(_lib.InvalidConfig):
        F.construct(F.blocked_bloomfilter_config(word_size=2), 1 << 16)
    with pytest.raises(_lib.InvalidConfig):
        F.cf(1 << 16, 6, 4)
    with pytest.raises(_lib.SizeError):
        F.bbf_32(1 << 40, 4)   # 2^35 blocks > 2^31 (block_addressing_logic.hpp:78-82)


def test_names_follow_reference_json():
    f = F.construct(F.blocked_bloomfilter_config(), 1024)
    assert f.name() == ('{"name":"blocked_bloom_multiword","size":128,"word_size":4,"k":8,"w":1,"s":1,'
                        '"u":0,"e":0,"addr":"pow2"}')
    z = F.zbbf_64(3000, 8, 8, 2)
    assert '"z":2' in z.name() and '"addr":"magic"' in z.name()
    c = F.cf(1 << 16, 16, 4)
    assert c.name().startswith('{"name":"cuckoo","size":8192,"tag_bits":16,"associativity":4')


def test_default_configs_match_reference():
    # blocked_bloomfilter_config.hpp:12-17, cuckoofilter_config.hpp:14-16
    c = F.blocked_bloomfilter_config()
    assert (c.k, c.word_size, c.word_cnt_per_block, c.sector_cnt, c.addr_mode, c.zone_cnt) == (8, 4, 1, 1, 0, 1)
    d = F.cuckoofilter_config()
    assert (d.bits_per_tag, d.tags_per_bucket, d.addr_mode) == (8, 2, 0)


@pytest.mark.parametrize("cfg,mib,plan", [
    # (word bytes, words, sectors, zones, k), filter MiB, expected automatic plan
    ((8, 8, 8, 1, 8), 128, 2), ((8, 8, 8, 1, 8), 168, 3), ((8, 8, 8, 1, 8), 512, 3),
    ((8, 4, 4, 1, 8), 192, 3),                       # 32-byte blocks: partitioned
    ((4, 1, 1, 1, 4), 168, 2), ((4, 1, 1, 1, 4), 256, 3),
    ((4, 16, 1, 1, 4), 224, 2), ((4, 16, 1, 1, 4), 256, 2), ((4, 16, 1, 1, 4), 384, 3),
    ((8, 8, 2, 1, 8), 192, 2),
    ((4, 16, 16, 2, 8), 192, 2), ((4, 16, 16, 2, 8), 256, 3),
    ((8, 8, 8, 2, 8), 256, 3), ((8, 8, 8, 4, 8), 192, 3),
])
def test_automatic_probe_plan(cfg, mib, plan):
    """The planner's choice for 2^28 probes (host logic only): the bitmask plan
    in block-range passes up to 160 MiB and, beyond, in the band of layouts it
    was measured faster for (s < w, one-word blocks, zoned u32); the
    partitioned plan (4 kernels: scatter, pair probe,
    overflow keys, compaction) otherwise.  Fewer than 2^20 keys: the fused
    single-kernel plan."""
    wb, w, s, z, k = cfg
    f = F.construct(F.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                 zone_cnt=z), mib << 23)
    L = _lib.lib()
    kernels = L.dtlg_probe_kernel_count(f._h, 1 << 28)
    assert (kernels == 4) == (plan == 3), (cfg, mib, kernels)
    assert L.dtlg_probe_kernel_count(f._h, (1 << 20) - 1) == 1
