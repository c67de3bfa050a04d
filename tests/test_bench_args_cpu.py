"""The benchmark's host-side helpers: workload variants from the command line
and the sector counts behind the cuckoo workloads' roofline numerator."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_cuckoo_bucket_sectors():
    # 4- and 8-byte buckets tile the 32-byte sectors; 2 of every 16 six-byte
    # buckets (byte offsets 28 and 30 mod 32) straddle a sector boundary
    assert bench.cuckoo_bucket_sectors(4) == 1.0
    assert bench.cuckoo_bucket_sectors(8) == 1.0
    assert bench.cuckoo_bucket_sectors(6) == 1.0 + 2 / 16
    assert bench.cuckoo_bucket_sectors(3) == 1.0 + 1 / 32 * 2


def test_layout_variant_of_a_bloom_workload(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "sectorized_l2", "--layout", "4,16,8,1,8",
                                      "--log2-build", "27"])
    args = bench.parse()
    assert args.workload == "sectorized_l2_n27_b16_h10_u32w16s8z1k8"
    assert bench.WORKLOADS[args.workload] == (4, 16, 8, 1, 8, 27, 16, 28, 0.10)
    cfg = bench.workload_config(args.workload, 1)
    assert cfg["filter"] == "blocked Bloom u32 w=16 s=8 z=1 k=8" and cfg["filter_bytes"] == (1 << 27) * 2


def test_layout_rejected_outside_bloom_workloads(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "cuckoo_dram", "--layout", "8,8,8,1,8"])
    with pytest.raises(SystemExit):
        bench.parse()
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "sectorized_l2", "--layout", "8,8"])
    with pytest.raises(SystemExit):
        bench.parse()


def test_host_chunks_mirror_the_pipeline():
    # chunks of 2^24 keys, the last 2^24 (or fewer) in four pieces
    assert bench.host_chunks(1 << 28) == [1 << 24] * 15 + [1 << 22] * 4
    assert bench.host_chunks(4) == [1, 1, 1, 1]
    assert bench.host_chunks(5) == [2, 2, 1]
    assert bench.host_chunks((1 << 24) * 2 + 12345) == [1 << 24] * 2 + [3087, 3087, 3087, 3084]
    for n in (1, 3, 1 << 24, (1 << 24) + 1, 123456789):
        assert sum(bench.host_chunks(n)) == n
