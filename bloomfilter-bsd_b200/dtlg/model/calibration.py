"""GPU calibration runs: probe cost per key of every candidate at every filter size.

The reference calibrates lookup costs per memory level on a few filter sizes
and interpolates with cache-miss probabilities (model/calibration.cpp:33-275,
cost_fn.hpp:80-145).  On the GPU the cost curve has more structure (L1, L2,
the TLB reach near 256 MiB, HBM), so each candidate is timed directly on a
grid of filter sizes and the cost model interpolates between grid points in
log2(bytes).

A probe tests the first half of a block (the first half of its words, or of
its zones / sectors) and loads the second half only when the first passes;
how often that happens depends on how full the filter is.  So every run
times two fills of the same filter:

* zeroed: every key fails on the first half -> ns_per_key, the first half;
* half-filled: the first half of every block all ones, the second half
  zeros -> every key passes the first half, loads the second and fails
  there; the difference is ns_second, the cost of the second half.

The cost model prices a filter at its bits per key from these two
(cost.py).  Layouts without a second part (blocks of one word, fixed-word
blocks under 64 bytes) show ns_second ~ 0.  Filters are probed with uniform
random uint32 keys through the public batch_contains path, timed with CUDA
events (median of `reps` launches after a warm-up).  The cost of a match
(writing its position) is measured on all-ones Bloom filters, where every key
matches, and reported as ns_per_match; the few keys a half-filled filter
matches (a layout whose bits can all fall in the first half) are charged at
that rate and taken out of ns_second.

    python -m dtlg.model.calibration --out calibration.npz   (needs a GPU)
"""
import argparse
import json
import os
import time
from dataclasses import dataclass, field

import numpy as np

from .candidates import all_candidates, by_name

DEFAULT_LOG2_BYTES = tuple(round(10 + 0.3 * i, 4) for i in range(71))   # 1 KiB .. 2 GiB
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DEFAULT_PATH = os.path.join(DATA_DIR, "calibration_b200.npz")


@dataclass
class CalibrationData:
    candidates: list            # [Candidate]
    log2_bytes: np.ndarray      # (S,) filter sizes of the grid
    ns_per_key: np.ndarray      # (C, S) probe time per key, zeroed filter (first half only)
    ns_per_match: float         # added cost per matching key
    meta: dict = field(default_factory=dict)
    ns_second: np.ndarray = None  # (C, S) added time per key that loads the second half

    def save(self, path):
        extra = {} if self.ns_second is None else {"ns_second": self.ns_second}
        np.savez_compressed(path, candidates=np.array([c.name for c in self.candidates]),
                            log2_bytes=self.log2_bytes, ns_per_key=self.ns_per_key,
                            ns_per_match=np.float64(self.ns_per_match), meta=json.dumps(self.meta), **extra)

    @staticmethod
    def load(path=DEFAULT_PATH):
        z = np.load(path, allow_pickle=False)
        sec = z["ns_second"].astype(np.float64) if "ns_second" in z.files else None
        return CalibrationData([by_name(str(n)) for n in z["candidates"]], z["log2_bytes"].astype(np.float64),
                               z["ns_per_key"].astype(np.float64), float(z["ns_per_match"]),
                               json.loads(str(z["meta"])), sec)

    def index(self, cand):
        return [c.name for c in self.candidates].index(cand.name)


def _magic_bits(nbytes, cand):
    """Filter size in bits near nbytes whose block count is not a power of two."""
    m = int(round(nbytes * 8))
    blk_bits = cand.block_bytes * 8 if cand.kind == "bloom" else cand.t * cand.b
    blocks = max(2, -(-m // blk_bits))
    if blocks & (blocks - 1) == 0:
        blocks += 1
    return blocks * blk_bits


class _Runner:
    def __init__(self, probe_cnt, max_bytes, seed, device):
        import torch

        from .. import _lib
        self.torch = torch
        self.L = _lib.lib()
        self.dev = torch.device(device)
        self.stream = torch.cuda.current_stream(self.dev)
        g = torch.Generator(device=self.dev)
        g.manual_seed(seed)
        self.keys = torch.randint(-2 ** 31, 2 ** 31, (probe_cnt,), dtype=torch.int32, device=self.dev, generator=g)
        self.arena = torch.zeros(int(max_bytes) // 8 + 64, dtype=torch.int64, device=self.dev)
        self.pos = torch.empty(probe_cnt, dtype=torch.int32, device=self.dev)
        self.cnt = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.ws = torch.empty(self.L.dtlg_probe_workspace_size(probe_cnt), dtype=torch.uint8, device=self.dev)
        self.ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def probe_ns_per_key(self, f, words, reps):
        import ctypes as C
        L = self.L
        n = self.keys.numel()
        args = (f._h, C.c_void_p(words.data_ptr()), C.c_void_p(self.keys.data_ptr()), n,
                C.c_void_p(self.pos.data_ptr()), 0, C.c_void_p(self.cnt.data_ptr()), C.c_void_p(self.ws.data_ptr()),
                self.ws.numel(), C.c_void_p(self.stream.cuda_stream))
        st = L.dtlg_batch_contains_ws(*args)  # warm-up
        if st != 0:
            raise RuntimeError(f"probe failed with status {st}")
        ts = []
        for _ in range(reps):
            self.ev[0].record(self.stream)
            L.dtlg_batch_contains_ws(*args)
            self.ev[1].record(self.stream)
            self.ev[1].synchronize()
            ts.append(self.ev[0].elapsed_time(self.ev[1]) * 1e6 / n)
        return float(np.median(ts)), int(self.cnt.item())


def _half_fill(arena, block_bytes):
    """The first half of every block-sized stretch of the arena all ones, the
    second half zeros (blocks of one word: all zeros)."""
    import torch
    b = arena.view(torch.uint8)
    pat = torch.zeros(block_bytes, dtype=torch.uint8, device=arena.device)
    if block_bytes >= 8:
        pat[: block_bytes // 2] = 0xFF
    reps = b.numel() // block_bytes
    b[: reps * block_bytes].view(reps, block_bytes).copy_(pat.expand(reps, block_bytes))
    b[reps * block_bytes:].zero_()


def run_calibration(candidates=None, log2_bytes=DEFAULT_LOG2_BYTES, probe_cnt=1 << 23, reps=3, seed=2024,
                    device="cuda", progress=True):
    """Time every candidate at every size, zeroed and half-filled; returns
    CalibrationData plus the run log (candidate, log2 bytes, m, ns zeroed, ns
    second half)."""
    import torch

    from .. import construct
    candidates = list(candidates or all_candidates())
    log2_bytes = np.asarray(log2_bytes, dtype=np.float64)
    max_bytes = max(_magic_bits(2.0 ** log2_bytes.max(), c) // 8 for c in candidates) + 4096
    R = _Runner(probe_cnt, max_bytes, seed, device)
    t_start = time.time()
    # the cost of a match first: all-ones Bloom filters match every key
    deltas = []
    blooms = [c for c in candidates if c.kind == "bloom"]
    for cand in blooms[::max(1, len(blooms) // 12)]:
        for lb in (16.0, 22.0, 26.0):
            m = _magic_bits(2.0 ** lb, cand)
            f = construct(cand.config(), m)
            words = R.arena[:max(1, f.alloc_words())]
            words.fill_(-1)
            ns1, cnt = R.probe_ns_per_key(f, words, reps)
            words.zero_()
            ns0, _ = R.probe_ns_per_key(f, words, reps)
            assert cnt == probe_cnt
            deltas.append(ns1 - ns0)
    ns_match = float(np.median(deltas))
    t = np.zeros((len(candidates), len(log2_bytes)))
    t2 = np.zeros((len(candidates), len(log2_bytes)))
    runs = []
    # zeroed runs
    R.arena.zero_()
    for ci, cand in enumerate(candidates):
        for si, lb in enumerate(log2_bytes):
            m = _magic_bits(2.0 ** lb, cand)
            f = construct(cand.config(), m)
            ns, cnt = R.probe_ns_per_key(f, R.arena[:max(1, f.alloc_words())], reps)
            if cnt != 0:
                raise RuntimeError(f"{cand.name}: zeroed filter matched {cnt} keys")
            t[ci, si] = ns
        if progress and (ci % 32 == 31 or ci == len(candidates) - 1):
            print(f"zeroed: {ci + 1}/{len(candidates)} candidates, {time.time() - t_start:.0f} s", flush=True)
    # half-filled runs, Bloom candidates grouped by block size (one fill each)
    for bb in sorted({c.block_bytes for c in blooms}):
        _half_fill(R.arena, bb)
        for ci, cand in enumerate(candidates):
            if cand.kind != "bloom" or cand.block_bytes != bb:
                continue
            for si, lb in enumerate(log2_bytes):
                m = _magic_bits(2.0 ** lb, cand)
                f = construct(cand.config(), m)
                ns, cnt = R.probe_ns_per_key(f, R.arena[:max(1, f.alloc_words())], reps)
                t2[ci, si] = max(0.0, ns - ns_match * cnt / probe_cnt - t[ci, si])
        if progress:
            print(f"half-filled: {bb}-byte blocks, {time.time() - t_start:.0f} s", flush=True)
    R.arena.zero_()
    for ci in range(len(candidates)):
        for si, lb in enumerate(log2_bytes):
            runs.append((ci, float(lb), _magic_bits(2.0 ** lb, candidates[ci]), t[ci, si], t2[ci, si]))
    props = torch.cuda.get_device_properties(R.dev)
    meta = {"device": props.name, "sms": props.multi_processor_count, "l2_bytes": getattr(props, "L2_cache_size", 0),
            "probe_keys": probe_cnt, "reps": reps, "seed": seed,
            "runs": len(runs) + int(np.sum([c.kind == "bloom" for c in candidates])) * len(log2_bytes)
            + 2 * len(deltas),
            "match_cost_runs": len(deltas), "api": "dtlg_batch_contains_ws (automatic probe plan)",
            "fills": "zeroed (first half of each block) and half-filled (second half of each block)",
            "keys": "uniform random uint32 (torch.randint)", "seconds": round(time.time() - t_start, 1),
            "date": time.strftime("%Y-%m-%d")}
    return CalibrationData(candidates, log2_bytes, t, ns_match, meta, t2), np.array(runs)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--probe-keys", type=int, default=1 << 23)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--quick", action="store_true", help="every 8th candidate, every 4th size")
    args = ap.parse_args()
    cands = all_candidates()
    sizes = DEFAULT_LOG2_BYTES
    if args.quick:
        cands, sizes = cands[::8], sizes[::4]
    data, runs = run_calibration(cands, sizes, args.probe_keys, args.reps)
    data.save(args.out)
    np.save(os.path.splitext(args.out)[0] + "_runs.npy", runs)
    print(json.dumps({"out": args.out, "candidates": len(cands), "sizes": len(sizes), **data.meta,
                      "ns_per_match": data.ns_per_match}))


if __name__ == "__main__":
    main()
