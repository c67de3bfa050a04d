"""Several GPUs, one process each (torch.distributed): sharded probes and
sharded Bloom builds.

Probe: the filter words are replicated (the reference replicates them per
NUMA node, filter.hpp:128-152) and each rank probes a contiguous slice of the
probe keys with match_offset = the slice's first index, so every rank's match
positions are already global and ascending; the only exchange is an
all-gather of the per-rank match counts (8 bytes each), which places each
rank's list in the concatenated result.

Build: each rank inserts its slice of the build keys into its own copy of
the words; the partial filters are OR-combined by block range (all-to-all of
word ranges, OR on the device with dtlg_or_words, all-gather of the ORed
ranges).  NCCL has no bitwise-OR reduction, hence the exchange.  Cuckoo
filters are not sharded (their kick chains are global): build on one rank and
broadcast the words.
"""
import ctypes as C

from ._lib import check, lib


def shard_bounds(total, rank, world):
    """(first index, count) of rank's contiguous share of `total` items."""
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def gather_counts(local_count, group=None):
    """All ranks' match counts, in rank order (all-gather of one int64)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    mine = torch.tensor([int(local_count)], dtype=torch.int64, device=dev)
    out = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(out, mine, group=group)
    return [int(t.item()) for t in out]


def output_offsets(counts):
    """Where each rank's positions start in the concatenated match list."""
    offs, acc = [], 0
    for c in counts:
        offs.append(acc)
        acc += c
    return offs, acc


def or_words(dst, srcs):
    """dst |= every tensor in srcs (int64 words of equal length): the
    library's kernel for CUDA tensors, torch for host tensors."""
    import torch
    if not srcs:
        return dst
    if dst.is_cuda:
        stack = torch.stack(list(srcs)).contiguous()
        check(lib().dtlg_or_words(C.c_void_p(dst.data_ptr()), C.c_void_p(stack.data_ptr()), dst.numel(),
                                  len(srcs), dst.numel(), C.c_void_p(torch.cuda.current_stream().cuda_stream)),
              "or_words")
    else:
        for s in srcs:
            dst.bitwise_or_(s)
    return dst


def or_combine(words, group=None):
    """OR the ranks' partial filter words into the full filter on every rank.
    Each rank ORs one block range of the words (all-to-all), then the ranges
    are all-gathered; 2 x the filter bytes cross the links per rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if world == 1:
        return words
    n = words.numel()
    chunk = -(-n // world)
    padded = torch.zeros(chunk * world, dtype=words.dtype, device=words.device)
    padded[:n] = words
    recv = torch.empty_like(padded)   # recv chunk j = rank j's copy of this rank's range
    dist.all_to_all_single(recv, padded, group=group)
    parts_in = list(recv.split(chunk))
    mine = parts_in[0].clone()
    or_words(mine, parts_in[1:])
    parts = [torch.empty(chunk, dtype=words.dtype, device=words.device) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    words.copy_(torch.cat(parts)[:n])
    return words
