"""The several-GPU plumbing on CPU: two gloo ranks shard a probe (contiguous
slices, match_offset = slice start, all-gather of counts) and a Bloom build
(partial filters OR-combined by block range; also the classic Bloom filter;
the blocked cuckoo filter is replicated and only its probe shards).  The filter work itself is the
oracle's (the CPU stand-in for each rank's GPU); what is checked is that the
sharded results equal the single-process ones."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    import sys
    for p in (os.path.join(ROOT, "bloomfilter-bsd_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import oracle as O
    from dtlg import keygen
    from dtlg.shard import gather_counts, or_combine, output_offsets, shard_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg, n, P = (8, 8, 8, 2, 8), 50000, 200001
        ob = O.Bloom(*cfg, n * 12 + 7)
        bk = keygen.build_keys(n, 17)
        # sharded build: this rank's slice of the build keys, then OR-combine
        b0, bn = shard_bounds(n, rank, world)
        part = ob.alloc()
        ob.insert(part, bk[b0:b0 + bn])
        words = torch.from_numpy(part.view(np.int64).copy())
        or_combine(words)
        full = ob.alloc()
        ob.insert(full, bk)
        build_ok = np.array_equal(words.numpy().view(np.uint64), full)
        # sharded probe: replicated words, slice with global positions
        pk, _ = keygen.probe_keys(n, P, 0.1, 17)
        p0, pn = shard_bounds(P, rank, world)
        mine = ob.batch_contains(full, pk[p0:p0 + pn], p0 + 1000)
        counts = gather_counts(len(mine))
        offs, total = output_offsets(counts)
        lists = [None] * world
        dist.all_gather_object(lists, mine.tolist())
        merged = np.concatenate([np.array(x, dtype=np.uint32) for x in lists])
        ref = ob.batch_contains(full, pk, 1000)
        # classic Bloom filter: OR-combined partial builds equal the full build
        oc = O.ClassicBloom(5, n * 10 + 3, True)
        cpart = oc.alloc()
        oc.insert(cpart, bk[b0:b0 + bn])
        cwords = torch.from_numpy(cpart.view(np.int64).copy())
        or_combine(cwords)
        cfull = oc.alloc()
        oc.insert(cfull, bk)
        classic_ok = np.array_equal(cwords.numpy().view(np.uint64), cfull)
        # blocked cuckoo: no OR-combine (a cuckoo build is not a union), so the
        # table is built once and replicated; the probe shards as above
        ox = O.BlockedCuckoo(n * 32, 64, 16, 4)
        xt = ox.alloc()
        ox.insert(xt, bk, seed=4)
        xmine = ox.batch_contains(xt, pk[p0:p0 + pn], p0)
        xl = [None] * world
        dist.all_gather_object(xl, xmine.tolist())
        xmerged = np.concatenate([np.array(x, dtype=np.uint32) for x in xl])
        bcf_ok = bool(np.array_equal(xmerged, ox.batch_contains(xt, pk, 0)))
        results[rank] = (build_ok, bool(np.array_equal(merged, ref)), total == len(ref),
                         offs[rank] == int(np.searchsorted(ref, p0 + 1000)), classic_ok, bcf_ok)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharded_build_and_probe_match_single_process(world):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        results = man.dict()
        mp.start_processes(_worker, args=(world, _free_port(), results), nprocs=world, join=True,
                           start_method="spawn")
        got = dict(results)
    assert sorted(got) == list(range(world))
    for rank, flags in got.items():
        assert all(flags), (rank, flags)


def test_shard_bounds_cover_everything():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "bloomfilter-bsd_b200"))
    from dtlg.shard import output_offsets, shard_bounds
    for total in (0, 1, 7, 1000003):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and sum(c for _, c in spans) == total
            assert all(spans[i][0] + spans[i][1] == spans[i + 1][0] for i in range(world - 1))
    assert output_offsets([3, 0, 5]) == ([0, 3, 3], 8)
