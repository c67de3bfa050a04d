#!/usr/bin/env python3
"""Probe throughput of the DTL filter path on B200 (and of the reference on the host).

Workload (default, "sectorized_dram"): the cache-sectorized blocked Bloom
filter of the reference -- 64-byte blocks of 8 x 64-bit words, one sector per
word, k = 8 (u64, w=8, s=8, k=8) -- at 16 bits per key: build n = 2^28 keys
(512 MiB of filter words, DRAM-resident), probe 2^28 u32 keys per GPU of which
10 % are members.  A step is one batch_contains over the 2^28 probe keys,
writing the ascending match positions.  Inputs (1 GiB keys + 512 MiB filter)
exceed the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line on rank 0.  Multi-GPU: one process per GPU (torchrun),
each rank probes its own 2^28-key slice of the probe stream against a
replicated filter (weak scaling; the only collectives are the barrier and the
max-over-ranks of the timings).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "bloomfilter-bsd_b200"))

WORKLOADS = {
    # name: (word_size, w, s, z, k, log2 n, bits/key, log2 probes, hit ratio)
    "sectorized_dram": (8, 8, 8, 1, 8, 28, 16, 28, 0.10),
    "sectorized_l2": (8, 8, 8, 1, 8, 22, 16, 28, 0.10),
    # the same filter type at 2^27 keys (256 MiB, still DRAM-resident) with
    # 2^26 probes: the case ncu captures run on
    "sectorized_dram_small": (8, 8, 8, 1, 8, 27, 16, 26, 0.10),
    "register_blocked": (4, 1, 1, 1, 4, 20, 16, 24, 0.10),
    # a 64 KiB filter (2^15 keys): L1-resident; --probe-mode 4 probes a copy
    # in every CTA's shared memory instead
    "sectorized_small": (8, 8, 8, 1, 8, 15, 16, 28, 0.10),
}
CUCKOO_WORKLOADS = {
    # name: (bits per tag, tags per bucket, log2 n, load factor, log2 probes, hit ratio)
    "cuckoo_dram": (16, 4, 26, 0.95, 28, 0.10),
    # the same with 12-bit tags (6-byte buckets, some straddle a 32-byte
    # sector) and 8-bit tags (4-byte buckets); 8-bit tags at load 0.93: with
    # 255 tag values the alternate buckets of a bucket are too few to place
    # 2^26 keys at 0.95
    "cuckoo_dram_t12": (12, 4, 26, 0.95, 28, 0.10),
    "cuckoo_dram_t8": (8, 4, 26, 0.93, 28, 0.10),
}
BCF_WORKLOADS = {
    # name: (block bytes, tag bits, associativity, log2 n, log2 m bits, log2 probes, hit ratio)
    # dtl::bcf's default config: 64-byte blocks of 8 buckets x 4 16-bit tags,
    # 256 MiB (DRAM-resident) at half of its slots
    "bcf_dram": (64, 16, 4, 26, 31, 28, 0.10),
    # the same at 128 MiB (still beyond the 126 MB L2) and 2^26 probes: the
    # case ncu captures run on
    "bcf_dram_small": (64, 16, 4, 25, 30, 26, 0.10),
}
CLASSIC_WORKLOADS = {
    # name: (k, log2 n, bits/key, log2 probes, hit ratio, MAGIC addressing)
    # the classic Bloom filter (bloomfilter_logic<u32, POW2>): k = 4 random
    # words per key, 8 MiB (L2-resident)
    "classic_l2": (4, 22, 16, 28, 0.10, False),
}
SEED = 20240601


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("dtlg", "reference"), default="dtlg")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(CUCKOO_WORKLOADS) + sorted(BCF_WORKLOADS)
                    + sorted(CLASSIC_WORKLOADS) + ["batched512"],
                    default="sectorized_dram")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-filters", type=int, default=512, help="batched512: number of filters")
    ap.add_argument("--batch-max-log2", type=int, default=24, help="batched512: log2 of the largest n / probes")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="sectorized_dram: skip the batched-vs-per-filter comparison the default line carries")
    ap.add_argument("--probe-mode", type=int, default=0,
                    help="0 auto, 1 fused, 2 bitmask + block-range passes, 3 partitioned, 4 shared-memory filter copy")
    ap.add_argument("--probe-passes", type=int, default=0, help="block-range passes of mode 2 (0 auto)")
    ap.add_argument("--build-mode", type=int, default=0,
                    help="Bloom build plan: 0 auto, 1 one kernel of atomic ORs, 2 keys grouped by block range")
    ap.add_argument("--log2-build", type=int, default=None, help="Bloom workloads: log2 of the build keys")
    ap.add_argument("--bits-per-key", type=int, default=None, help="Bloom workloads: filter bits per build key")
    ap.add_argument("--hit-ratio", type=float, default=None, help="Bloom workloads: fraction of member probes")
    ap.add_argument("--layout", default=None,
                    help="Bloom workloads: the filter layout as WORD_BYTES,W,S,Z,K (e.g. 4,16,8,1,8 = u32 words, "
                         "16 per block, 8 sectors, 1 zone, k=8)")
    args = ap.parse_args()
    overrides = (args.log2_build, args.bits_per_key, args.hit_ratio, args.layout)
    if any(v is not None for v in overrides):
        # a variant of a Bloom workload (the shapes of the sectorized config:
        # n in {2^22, 2^26, 2^28}, 8/12/16 bits per key, 1/10/50 % hits)
        if args.workload not in WORKLOADS:
            ap.error("--log2-build / --bits-per-key / --hit-ratio / --layout apply to Bloom workloads only")
        wb, w, s_, z, k, ln, bpk, lp, hit = WORKLOADS[args.workload]
        ln = ln if args.log2_build is None else args.log2_build
        bpk = bpk if args.bits_per_key is None else args.bits_per_key
        hit = hit if args.hit_ratio is None else args.hit_ratio
        name = f"{args.workload}_n{ln}_b{bpk}_h{round(hit * 100)}"
        if args.layout is not None:
            try:
                wb, w, s_, z, k = (int(v) for v in args.layout.split(","))
            except ValueError:
                ap.error("--layout takes WORD_BYTES,W,S,Z,K")
            name += f"_u{wb * 8}w{w}s{s_}z{z}k{k}"
        WORKLOADS[name] = (wb, w, s_, z, k, ln, bpk, lp, hit)
        args.workload = name
    return args


def cuckoo_bits(n, t, b, lf):
    """Table size in bits for n keys at load factor lf whose MAGIC bucket count
    is odd: with an even one the reference's two-choice insert stalls near 75 %
    occupancy (cuckoofilter_logic.hpp:216-252)."""
    import dtlg
    b0 = int(-(-n // (b * lf)))
    for i in range(4096):
        m = (b0 + i) * t * b
        f = dtlg.cf(m, t, b)
        if f.block_cnt() % 2 == 1 and f.is_magic() and f.block_cnt() * b * lf >= n:
            return m
    raise RuntimeError("no odd MAGIC bucket count found")


def host_chunks(n, chunk=1 << 24):
    """Key counts of the pieces dtlg_batch_contains_host streams n keys in
    (csrc/host_pipeline.cu): chunks of 2^24 keys, the last 2^24 keys or fewer
    in four pieces."""
    full = (n - 1) // chunk if n > chunk else 0
    tail = n - full * chunk
    piece = max(1, -(-tail // 4))
    return [chunk] * full + [min(piece, tail - i) for i in range(0, tail, piece)]


def cuckoo_bucket_sectors(bucket_bytes):
    """Mean 32-byte sectors one bucket of a packed cuckoo table touches: 1
    when buckets tile the sectors (4 or 8 bytes), more when some straddle a
    sector boundary (6-byte buckets: 2 of every 16 do)."""
    period = 32 // math.gcd(32, bucket_bytes)
    return sum(1 + ((bucket_bytes * i) % 32 + bucket_bytes > 32) for i in range(period)) / period


def bcf_sectors(block_bytes, t, a):
    """Distinct 32-byte sectors a blocked cuckoo probe reads: its two bucket
    words lie in one block; x = i1 ^ i2 is uniform over the block's buckets,
    and both words share a sector iff x < buckets per sector."""
    word = 4 if t * a <= 32 else 8
    per_block = block_bytes // word
    if block_bytes <= 32:
        return 1.0
    return 2.0 - (32 // word) / per_block


def workload_config(name, n_gpus):
    if name in CLASSIC_WORKLOADS:
        k, ln, bpk, lp, h, magic = CLASSIC_WORKLOADS[name]
        return {
            "workload": name, "filter": f"classic Bloom (bloomfilter_logic) k={k} {'MAGIC' if magic else 'POW2'}",
            "bits_per_key": bpk, "build_keys": 1 << ln, "probe_keys_per_gpu": 1 << lp,
            "global_batch": (1 << lp) * n_gpus, "hit_ratio": h, "filter_bytes": (1 << ln) * bpk // 8,
            "parallelism": f"dp{n_gpus} (replicated filter, sharded probes)",
            "l2_flush": "inputs larger than L2 (keys 4 B/key x probes + filter words)",
        }
    if name in BCF_WORKLOADS:
        bb, t, a, ln, lm, lp, h = BCF_WORKLOADS[name]
        return {
            "workload": name, "filter": f"blocked cuckoo (dtl::bcf) block={bb} B t={t} a={a}",
            "build_keys": 1 << ln, "probe_keys_per_gpu": 1 << lp, "global_batch": (1 << lp) * n_gpus,
            "hit_ratio": h, "filter_bytes": (1 << lm) // 8,
            "parallelism": f"dp{n_gpus} (replicated filter, sharded probes)",
            "l2_flush": "inputs larger than L2 (keys 4 B/key x probes + filter words)",
        }
    if name in CUCKOO_WORKLOADS:
        t, b, ln, lf, lp, h = CUCKOO_WORKLOADS[name]
        return {
            "workload": name, "filter": f"cuckoo t={t} b={b} (MAGIC, odd bucket count)", "load_factor": lf,
            "build_keys": 1 << ln, "probe_keys_per_gpu": 1 << lp, "global_batch": (1 << lp) * n_gpus,
            "hit_ratio": h, "filter_bytes": int(-(-(1 << ln) // (b * lf))) * t * b // 8,
            "parallelism": f"dp{n_gpus} (replicated filter, sharded probes)",
            "l2_flush": "inputs larger than L2 (keys 4 B/key x probes + filter words)",
        }
    wb, w, s, z, k, ln, bpk, lp, h = WORKLOADS[name]
    return {
        "workload": name,
        "filter": f"blocked Bloom u{wb * 8} w={w} s={s} z={z} k={k}",
        "bits_per_key": bpk, "build_keys": 1 << ln, "probe_keys_per_gpu": 1 << lp,
        "global_batch": (1 << lp) * n_gpus, "hit_ratio": h,
        "filter_bytes": (1 << ln) * bpk // 8, "parallelism": f"dp{n_gpus} (replicated filter, sharded probes)",
        "l2_flush": "inputs larger than L2 (keys 4 B/key x probes + filter words)",
    }


# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and throttle reasons during the timed region.  NVML is polled
    every 2 ms in a thread and the samples between mark_start() and mark_end()
    are kept (a 20-step timed region lasts only tens of ms).  Without NVML,
    nvidia-smi -lms 100 samples from start() to stop() instead.  Reads only."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    # NVML clocks-event reason bits of the same four (nvml.h)
    NVML_BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, gpu_index, nvml=None):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.nvml = nvml            # the NVML module (pynvml unless given)
        self._nv = None
        self.thread = None
        self.samples = []           # (perf_counter, sm MHz, reason bits)
        self.t0 = self.t1 = None
        self.max_mhz = None
        self.stop_evt = threading.Event()

    def start(self):
        if not self._start_nvml():
            self._start_smi()

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()

    def _start_nvml(self):
        try:
            nv = self.nvml
            if nv is None:
                import pynvml as nv
            nv.nvmlInit()
            try:
                import torch
                p = torch.cuda.get_device_properties(self.gpu)
                h = nv.nvmlDeviceGetHandleByPciBusId(
                    f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0")
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._reasons = (getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None)
                             or nv.nvmlDeviceGetCurrentClocksThrottleReasons)
            self._nv, self._h = nv, h
            self._poll()            # a failing query fails here, not in the thread
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
            return True
        except Exception:
            self._nv = None
            return False

    def _poll(self):
        t = time.perf_counter()
        sm = float(self._nv.nvmlDeviceGetClockInfo(self._h, self._nv.NVML_CLOCK_SM))
        self.samples.append((t, sm, int(self._reasons(self._h))))

    def _run(self):
        while not self.stop_evt.wait(0.002):
            try:
                self._poll()
            except Exception:
                return

    def _start_smi(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_evt.set()
            self.thread.join(timeout=2)
            try:
                self._nv.nvmlShutdown()
            except Exception:
                pass
            done = list(self.samples)
            win = [x for x in done if self.t0 is not None and self.t1 is not None and self.t0 <= x[0] <= self.t1]
            used = win or done
            reasons = {nm for nm, bit in self.NVML_BITS.items() for _, _, r in used if r & bit}
            return {"sm_mhz": statistics.median(x[1] for x in used), "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(reasons), "samples": len(used),
                    "source": "NVML every 2 ms, " + ("timed region" if win else "whole run")}
        return self._stop_smi()

    def _stop_smi(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi every 100 ms, whole run"}


def load_traffic_profile():
    """DRAM bytes per probed key of one probe step, per workload, from the
    committed ncu summary (profiles/probe_traffic.json)."""
    path = os.path.join(ROOT, "profiles", "probe_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except OSError:
        return None


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured: MEASURED_PEAKS.json hbm_gbs"
    except Exception:
        return 6650.0, "fallback: 6.65 TB/s copy bandwidth measured earlier on this GPU type (no MEASURED_PEAKS.json)"


# ---------------------------------------------------------------------------
# The reference's CPU path, one method for both arms: the reference's own
# batch_contains (oracle/_ref: its filter logic compiled from its sources) on
# all host threads, each thread on its own contiguous slice in 1024-key batches
# (model/benchmark.cpp:123-165, batchwise.hpp:9), with the SIMD unroll factor
# the reference's own calibration picks (blocked_bloomfilter_tune_impl.hpp:
# 162-256, cuckoofilter_tune_impl.hpp:118-225).  The sample is the first
# REF_SAMPLE keys of the workload's probe stream; the statistic is keys over
# the summed time of the timed runs (the mean rate).
REF_SAMPLE = 1 << 26


class RefProbe:
    """The reference's probe of one workload's filter on the host."""

    def __init__(self, cfg, m, words_np, threads):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import numpy as np

        import oracle as O
        self.threads = threads
        self.unroll, self.unroll_ns = None, None
        if cfg[0] in ("classic", "bcf"):
            ref = O.try_refcbf() if cfg[0] == "classic" else bcf_reference()
            if ref is None:
                raise RuntimeError(f"the reference's {cfg[0]} filter is not built (oracle/_ref)")
            f = ref.create(cfg[1], m, cfg[2]) if cfg[0] == "classic" else ref.create(m, cfg[1], cfg[2], cfg[3])
            words = np.zeros(f.size_u32 + 16, dtype=np.uint32)
            words[: f.size_u32] = words_np.view(np.uint32)[: f.size_u32]
            self.variant = "scalar" if cfg[0] == "classic" else ref.variant
            # neither has an unroll parameter (bcf.cpp, bloomfilter_logic.hpp)
            self._count = lambda keys, out: f.batch_contains_mt(words, keys, threads, out=out)  # noqa: E731
            self._list = lambda keys, out: f.batch_contains_mt_list(words, keys, threads, out=out)  # noqa: E731
        else:
            ref = O.try_reflib()
            if ref is None:
                raise RuntimeError("the reference's filter logic is not built (oracle/_ref)")
            f = ref.cuckoo(cfg[1], cfg[2], m) if cfg[0] == "cuckoo" else ref.bloom(*cfg, m)
            if f is None:
                raise RuntimeError("this configuration is not instantiated in oracle/_ref")
            words = words_np
            self.variant = f"{ref.variant}, {ref.lanes} lanes"
            self.unroll, per = f.calibrate_unroll(words, cuckoo=cfg[0] == "cuckoo")
            self.unroll_ns = {str(u): round(v, 3) for u, v in per.items()}
            u = self.unroll
            self._count = lambda keys, out: f.batch_contains_mt(words, keys, threads, unroll=u, out=out)  # noqa: E731
            self._list = lambda keys, out: f.batch_contains_mt_list(words, keys, threads, unroll=u, out=out)  # noqa: E731

    def rate(self, probe_np, runs, warmup=1):
        """(keys/s, sample keys, count, seconds per run) over the sample."""
        import numpy as np
        n = min(len(probe_np), REF_SAMPLE)
        out = np.empty(n + 64, dtype=np.uint32)
        keys = probe_np[:n]
        for _ in range(max(1, warmup)):
            self._count(keys, out)
        total, cnt = 0.0, 0
        for _ in range(max(1, runs)):
            t0 = time.perf_counter()
            cnt = self._count(keys, out)
            total += time.perf_counter() - t0
        return n * runs / total, n, int(cnt), total / runs

    def positions(self, probe_np):
        """The reference's whole ascending match list of these keys."""
        import numpy as np
        out = np.empty(len(probe_np) + 64, dtype=np.uint32)
        return self._list(probe_np, out)

    def describe(self):
        u = "" if self.unroll is None else f", unroll u={self.unroll} (the reference's calibration)"
        return (f"{self.threads} threads x 1024-key batches (model/benchmark.cpp:123-165), "
                f"the reference's batch_contains ({self.variant}{u})")


def l2_gather_peak(L, words, nbytes, stream, n_sectors=1 << 28, steps=5):
    """Random 32-byte sector gathers from `words` (GB/s of sectors), timed with
    CUDA events on `stream` after 3 warm-up launches."""
    import ctypes as C
    import torch
    sink = torch.zeros(1, dtype=torch.int64, device=words.device)

    def run():
        st = L.dtlg_sector_gather(C.c_void_p(words.data_ptr()), nbytes, n_sectors, C.c_void_p(sink.data_ptr()),
                                  C.c_void_p(stream.cuda_stream))
        if st:
            raise RuntimeError(f"dtlg_sector_gather failed: {st}")
    for _ in range(3):
        run()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        run()
    b.record(stream)
    torch.cuda.synchronize()
    return n_sectors * 32 / (a.elapsed_time(b) / steps / 1e3) / 1e9


def spread_copy(a, threads):
    """A copy of `a` whose pages are first touched by `threads` threads, one
    contiguous slice each: on a host with several memory nodes the pages land
    spread over them, as those of a filter and key set that many threads built
    (an array copied from the GPU by one thread sits on one node, and the
    probes of every thread on another node then read remote memory)."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor
    out = np.empty_like(a)
    step = -(-len(a) // max(1, threads))

    def part(i):
        out[i:i + step] = a[i:i + step]
    with ThreadPoolExecutor(max(1, threads)) as ex:
        list(ex.map(part, range(0, len(a), step)))
    return out


def list_checksum(pos):
    """Order-sensitive checksum of a position list: sum of pos[i] * (2i + 1)
    mod 2^64 (any reordering, loss or change of a position changes it)."""
    import numpy as np
    total = np.uint64(0)
    for b in range(0, len(pos), 1 << 24):
        p = np.asarray(pos[b:b + (1 << 24)], dtype=np.uint64)
        w = np.arange(2 * b + 1, 2 * (b + len(p)) + 1, 2, dtype=np.uint64)
        total = total + (p * w).sum(dtype=np.uint64)
    return int(total)


def bcf_reference():
    """The reference's dtl::bcf (oracle/_ref): its AVX2 build where the host
    has AVX2 (the build a user compiling for this host runs), else scalar."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if "avx2" in O._cpu_flags():
        r = O.try_refbcf("avx2")
        if r is not None:
            return r
    return O.try_refbcf("scalar")


# ---------------------------------------------------------------------------
def run_dtlg(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import dtlg
    from dtlg import keygen

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    if args.workload in CUCKOO_WORKLOADS:
        tag_bits, slots, ln, lf, lp, hit = CUCKOO_WORKLOADS[args.workload]
        n_build, P = 1 << ln, 1 << lp
        m = cuckoo_bits(n_build, tag_bits, slots, lf)
        f = dtlg.cf(m, tag_bits, slots)
        block_bytes = (tag_bits * slots + 7) // 8
        sectors = 2 * cuckoo_bucket_sectors(block_bytes)   # two buckets
    elif args.workload in CLASSIC_WORKLOADS:
        ck, ln, bpk, lp, hit, cmagic = CLASSIC_WORKLOADS[args.workload]
        n_build, P = 1 << ln, 1 << lp
        m = n_build * bpk
        f = dtlg.bloomfilter_logic(m, ck, dtlg.MAGIC if cmagic else dtlg.POWER_OF_TWO)
        sectors = ck   # k words anywhere in the filter: one sector each (members; non-members stop earlier)
    elif args.workload in BCF_WORKLOADS:
        block_bytes, tag_bits, assoc, ln, lm, lp, hit = BCF_WORKLOADS[args.workload]
        n_build, P = 1 << ln, 1 << lp
        m = 1 << lm
        f = dtlg.bcf(m, block_bytes, tag_bits, assoc)
        sectors = bcf_sectors(block_bytes, tag_bits, assoc)
    else:
        wb, w, s, z, k, ln, bpk, lp, hit = WORKLOADS[args.workload]
        n_build, P = 1 << ln, 1 << lp
        m = n_build * bpk
        cfg = dtlg.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s, zone_cnt=z)
        f = dtlg.construct(cfg, m)
        block_bytes = w * wb
        sectors = -(-block_bytes // 32)
    f.set_probe_options(args.probe_mode, -1)
    f.set_probe_passes(args.probe_passes)
    f.set_build_options(args.build_mode)
    words = f.alloc_filter_data()
    bk = keygen.build_keys_torch(n_build, SEED)
    assert f.batch_insert(words, bk), "build failed"
    # build throughput (setup, not the metric): a second build into zeroed words
    torch.cuda.synchronize()
    words.zero_()
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record()
    assert f.batch_insert(words, bk), "build failed"
    b1.record()
    torch.cuda.synchronize()
    build_ms = b0.elapsed_time(b1)
    if args.workload in CUCKOO_WORKLOADS:
        occupied = f.count_occupied_slots(words)
        assert occupied == n_build, (occupied, n_build)
    del bk
    # this rank's slice of the probe stream; positions are global (offset)
    start = rank * P
    keys, member = keygen.probe_keys_torch(n_build, P, hit, SEED, start=start)
    n_members = int(member.sum().item())
    del member
    out = torch.empty(P, dtype=torch.int32, device="cuda")
    cnt_dev = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws_bytes = dtlg.lib().dtlg_probe_workspace_size(P)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    L = dtlg.lib()
    import ctypes as C

    def step():
        st = L.dtlg_batch_contains_ws(f._h, C.c_void_p(words.data_ptr()), C.c_void_p(keys.data_ptr()), P,
                                      C.c_void_p(out.data_ptr()), start & 0xFFFFFFFF, C.c_void_p(cnt_dev.data_ptr()),
                                      C.c_void_p(ws.data_ptr()), ws_bytes, C.c_void_p(stream.cuda_stream))
        if st:
            raise RuntimeError(f"dtlg_batch_contains_ws failed: {st}")

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    count = int(cnt_dev.item())
    # correctness of the bench's own output: every member found, positions in range
    assert count >= n_members, (count, n_members)
    # the GPU's whole match list, checked against the reference's after timing
    check_parity = rank == 0 and world == 1 and not args.no_cpu_baseline
    gpu_positions = out[:count].cpu().numpy().view(np.uint32).copy() if check_parity else None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    clocks.mark_start()
    t_start.record(stream)
    for i in range(args.steps):
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    clocks.mark_end()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    per_launch_ms = [a.elapsed_time(b) for a, b in evs]
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * P / (ms_per_step / 1e3) / 1e9  # Gkeys/s, whole job

    # roofline of the probe kernel (one launch per step)
    mu = count / P
    dram_resident = f.size_in_bytes() > torch.cuda.get_device_properties(local).L2_cache_size
    S = sectors if dram_resident else 0
    alg_bytes_per_key = 4 + 4 * mu + 32 * S
    launch_ms = statistics.mean(per_launch_ms)
    achieved = P * alg_bytes_per_key / (launch_ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    prof = load_traffic_profile()
    traffic = None
    if prof and isinstance(prof.get(args.workload), dict) and args.probe_mode == 0 and args.probe_passes == 0:
        traffic = round(prof[args.workload]["dram_bytes_per_key"] * P)

    # an L2-resident filter moves no filter bytes from HBM: its probe is bounded
    # by the random-sector gather rate from L2, measured here over the filter's
    # own words with the probe's load instruction (dtlg_sector_gather)
    roofline_l2 = None
    if not dram_resident:
        gather_peak = l2_gather_peak(L, words, f.size_in_bytes(), stream)
        l2_achieved = P * 32 * sectors / (launch_ms / 1e3) / 1e9
        roofline_l2 = {"bound": "l2", "achieved": round(l2_achieved, 1), "peak": round(gather_peak, 1), "unit": "GB/s",
                       "frac": round(l2_achieved / gather_peak, 4),
                       "algorithmic_bytes_per_key": 32 * sectors,
                       "peak_source": "measured in this run: dtlg_sector_gather, 2^28 random 32-byte sectors of the "
                                      "filter's words, one 256-bit load each"}

    result = {
        "metric": "probe Gkeys/s (batch_contains, ascending match positions)",
        "value": round(value, 3), "unit": "Gkeys/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic: seeded u32 bijection keys (no dataset is published for this path)",
        "config": workload_config(args.workload, world),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_key": round(alg_bytes_per_key, 3),
                     "dram_resident": dram_resident},
        "roofline_l2": roofline_l2,
        "gpu_launches": args.steps * L.dtlg_probe_kernel_count(f._h, P),
        "kernels_per_step": L.dtlg_probe_kernel_count(f._h, P),
        "match_count_per_gpu": count,
        "clocks": clk,
        "build": {"ms": round(build_ms, 3), "gkeys_s": round(n_build / (build_ms / 1e3) / 1e9, 3),
                  "api": "dtlg_batch_insert (device keys), second build into zeroed words, not in the metric"},
    }

    # end to end through the public host-buffer API (pinned keys in, positions out)
    if not args.no_e2e:
        keys_h = torch.empty(P, dtype=torch.int32, pin_memory=True)
        keys_h.copy_(keys)
        pos_h = torch.empty(P, dtype=torch.int32, pin_memory=True)
        out = None
        torch.cuda.empty_cache()
        cnt = C.c_uint64(0)

        def e2e_step():
            st = L.dtlg_batch_contains_host(f._h, C.c_void_p(words.data_ptr()), C.c_void_p(keys_h.data_ptr()), P,
                                            C.c_void_p(pos_h.data_ptr()), start & 0xFFFFFFFF, C.byref(cnt),
                                            C.c_void_p(stream.cuda_stream))
            if st:
                raise RuntimeError(f"dtlg_batch_contains_host failed: {st}")

        e2e_step()
        torch.cuda.synchronize()
        assert cnt.value == count
        e_steps = max(3, min(args.steps, 10))
        if world > 1:
            dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(e_steps):
            e2e_step()
        b.record(stream)
        torch.cuda.synchronize()
        et = torch.tensor([a.elapsed_time(b) / e_steps], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        e_ms = float(et.item())
        chunks = host_chunks(P)
        # the bound of the host-buffer path: one plain copy of the same pinned
        # keys to the device (median of 3), the PCIe host-to-device rate
        dst = torch.empty_like(keys)
        h2d = []
        for _ in range(3):
            a.record(stream)
            dst.copy_(keys_h, non_blocking=True)
            b.record(stream)
            torch.cuda.synchronize()
            h2d.append(P * 4 / (a.elapsed_time(b) / 1e3) / 1e9)
        del dst
        h2d_gbs = sorted(h2d)[1]
        result["e2e"] = {"value": round(world * P / (e_ms / 1e3) / 1e9, 3), "unit": "Gkeys/s",
                         "ms_per_step": round(e_ms, 3), "h2d_bytes_per_step": P * 4,
                         "d2h_bytes_per_step": count * 4 + 8 * len(chunks),
                         "api": "dtlg_batch_contains_host (pinned host keys -> host positions)",
                         "pcie_h2d_gbs": round(h2d_gbs, 2),
                         "frac_of_pcie_h2d": round(P * 4 / (e_ms / 1e3) / 1e9 / h2d_gbs, 4)}
        result["gpu_launches"] += e_steps * sum(L.dtlg_probe_kernel_count(f._h, c) for c in chunks)

    # the reference's CPU path on this host (rank 0, N=1 only): its rate on a
    # bounded sample, and its whole match list of the same 2^28 keys against
    # the same filter words, compared with the GPU's list
    if check_parity:
        try:
            threads = len(os.sched_getaffinity(0))
            words_np = spread_copy(words.cpu().numpy().view(np.uint64), threads)
            probe_np = spread_copy(keys.cpu().numpy().view(np.uint32), threads)
            if args.workload in CUCKOO_WORKLOADS:
                fcfg = ("cuckoo", tag_bits, slots)
            elif args.workload in BCF_WORKLOADS:
                fcfg = ("bcf", block_bytes, tag_bits, assoc)
            elif args.workload in CLASSIC_WORKLOADS:
                fcfg = ("classic", ck, cmagic)
            else:
                fcfg = (wb, w, s, z, k)
            rp = RefProbe(fcfg, m, words_np, threads)
            rate, n, c, _ = rp.rate(probe_np, runs=5)
            result["cpu_baseline"] = {"value": round(rate / 1e9, 4), "unit": "Gkeys/s", "cores": threads,
                                      "kind": "reference",
                                      "sample": f"first {n} probe keys of this workload, mean of 5 runs, "
                                                + rp.describe(),
                                      "unroll": rp.unroll, "unroll_ns_per_key": rp.unroll_ns,
                                      "match_count": c}
            ref_positions = rp.positions(probe_np)
            same = len(ref_positions) == len(gpu_positions) and bool(np.array_equal(ref_positions, gpu_positions))
            result["parity"] = same
            result["parity_check"] = {
                "keys": P, "gpu_count": int(len(gpu_positions)), "reference_count": int(len(ref_positions)),
                "gpu_checksum": list_checksum(gpu_positions), "reference_checksum": list_checksum(ref_positions),
                "checksum": "sum of pos[i] * (2i + 1) mod 2^64 over the whole ascending list",
                "method": "the reference's batch_contains over every probe key of this step, same filter words"}
        except Exception as e:  # the baseline is reported, never required
            result["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
            result["parity"] = None

    # the metric's second half, batched vs per-filter launches (BASELINE's
    # 512-filter configuration), on the same GPU after the probe workload
    if world == 1 and args.workload == "sectorized_dram" and not args.no_batched:
        words = keys = ws = out = None
        torch.cuda.empty_cache()
        br = batched_bench(args)
        result["batched"] = {
            "workload": "batched512", "filters": br["config"]["filters"],
            "build_keys_total": br["config"]["build_keys_total"],
            "probe_keys_total": br["config"]["probe_keys_total"],
            "ms_batched": br["ms_per_step"], "ms_per_filter": br["per_filter"]["ms_per_step"],
            "speedup_vs_per_filter": br["speedup_vs_per_filter"],
            "probe_gkeys_s_batched": br["value"], "kernels_batched": br["gpu_launches"] // br["steps"],
            "kernels_per_filter": br["per_filter"]["kernels_per_step"],
            "bit_exact_vs_per_filter": br["bit_exact_vs_per_filter"], "steps": br["steps"],
            "step": br["config"]["step"]}
        result["gpu_launches"] += br["gpu_launches"]

    if world > 1:
        # the probe's one exchange: every rank's match count (places its
        # positions in the concatenated list)
        from dtlg.shard import gather_counts, output_offsets
        counts = gather_counts(count)
        result["match_count_total"] = output_offsets(counts)[1]
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """The reference's own CPU implementation of the path, same workload /
    metric, rank 0 only: the filter is built by the reference's insert
    (oracle/_ref: its filter logic, dtl::bcf or bloomfilter_logic compiled from
    its sources) and each step is one probe of the same sample as the GPU
    arm's cpu_baseline (RefProbe: all host threads, the reference's calibrated
    unroll factor)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from concurrent.futures import ThreadPoolExecutor

    from dtlg import keygen
    threads = len(os.sched_getaffinity(0))
    chunk = 1 << 24

    def unavailable(why):
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)

    if args.workload in BCF_WORKLOADS or args.workload in CLASSIC_WORKLOADS:
        if args.workload in CLASSIC_WORKLOADS:
            ck, ln, bpk, lp, hit, cmagic = CLASSIC_WORKLOADS[args.workload]
            ref, m, fcfg = O.try_refcbf(), (1 << ln) * bpk, ("classic", ck, cmagic)
        else:
            bb, t, a, ln, lm, lp, hit = BCF_WORKLOADS[args.workload]
            ref, m, fcfg = bcf_reference(), 1 << lm, ("bcf", bb, t, a)
        if ref is None:
            return unavailable("oracle/_ref (the reference compiled from its sources) is not built here")
        f = ref.create(ck, m, cmagic) if fcfg[0] == "classic" else ref.create(m, bb, t, a)
        words_u32 = f.alloc()
        n_build, P = 1 << ln, 1 << lp
        for c0 in range(0, n_build, chunk):   # their inserts are not atomic: one thread
            f.insert(words_u32, keygen.build_keys(min(chunk, n_build - c0), SEED, start=c0))
        words = np.zeros((len(words_u32) + 1) // 2 + 8, dtype=np.uint64)
        words.view(np.uint32)[: len(words_u32)] = words_u32
    else:
        ref = O.try_reflib()
        if ref is None:
            return unavailable("oracle/_ref (the reference compiled from its sources) is not built here")
        if args.workload in CUCKOO_WORKLOADS:
            t, b, ln, lf, lp, hit = CUCKOO_WORKLOADS[args.workload]
            m = cuckoo_bits(1 << ln, t, b, lf)
            f, fcfg, wbytes = ref.cuckoo(t, b, m), ("cuckoo", t, b), 4
        else:
            wb, w, s, z, k, ln, bpk, lp, hit = WORKLOADS[args.workload]
            m = (1 << ln) * bpk
            f, fcfg, wbytes = ref.bloom(wb, w, s, z, k, m), (wb, w, s, z, k), wb
        if f is None:
            return unavailable("this configuration is not instantiated in the reference build (oracle/_ref)")
        n_build, P = 1 << ln, 1 << lp
        # filter words plus (cuckoo) the victim record the reference keeps after them
        words = np.zeros((f.word_cnt * wbytes + 64) // 8, dtype=np.uint64)
        with ThreadPoolExecutor(max(1, min(threads, 32))) as ex:
            bk = np.concatenate(list(ex.map(lambda c0: keygen.build_keys(min(chunk, n_build - c0), SEED, start=c0),
                                            range(0, n_build, chunk))))
        if fcfg[0] == "cuckoo":
            assert f.insert(words, bk), "reference cuckoo build failed"   # its inserts are not thread-safe
        elif fcfg[3] == 1:
            f.insert_mt(words, bk, threads)    # CAS-based, thread-safe (..._sgew.hpp:300-325)
        else:
            f.insert(words, bk)                # zoned inserts are not atomic
        del bk
    with ThreadPoolExecutor(max(1, min(threads, 32))) as ex:
        probe = np.concatenate(list(ex.map(
            lambda c0: keygen.probe_keys(n_build, min(chunk, P - c0), hit, SEED, start=c0)[0],
            range(0, min(P, REF_SAMPLE), chunk))))
    rp = RefProbe(fcfg, m, words, threads)
    rate, n, cnt, sec = rp.rate(probe, runs=args.steps, warmup=args.warmup)
    value = rate / 1e9
    print(json.dumps({
        "impl": "reference", "metric": "probe Gkeys/s (batch_contains, ascending match positions)",
        "value": round(value, 4), "unit": "Gkeys/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic: seeded u32 bijection keys",
        "config": workload_config(args.workload, world),
        "cpu_baseline": {"value": round(value, 4), "unit": "Gkeys/s", "cores": threads, "kind": "reference",
                         "sample": f"first {n} probe keys of this workload per step, mean over the steps, "
                                   + rp.describe(),
                         "unroll": rp.unroll, "unroll_ns_per_key": rp.unroll_ns, "match_count": cnt},
        "e2e": {"value": round(value, 4), "unit": "Gkeys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


BATCH_CONFIGS = [(8, 8, 8, 2, 8), (8, 8, 8, 4, 8), (4, 16, 16, 2, 8), (4, 16, 16, 4, 8), (8, 8, 8, 1, 8)]


def batched_plan(n_filters=512, seed=4242, max_log2=24):
    """512 filters: config from the zoned (2/4 zones, u64 w=8 and u32 w=16) and
    sectorized (u64 w=8 s=8) set, n log-uniform over 2^10..2^24, probes
    log-uniform over 2^12..2^24 at 5 % hits, 8/12/16 bits per key (a smaller
    n_filters / max_log2 gives the small case that profilers capture)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    plan = []
    for i in range(n_filters):
        cfg = BATCH_CONFIGS[int(rng.integers(0, len(BATCH_CONFIGS)))]
        n = int(2 ** rng.uniform(10, max_log2))
        p = int(2 ** rng.uniform(12, max_log2))
        bpk = int(rng.choice([8, 12, 16]))
        plan.append((cfg, n * bpk, n, p))
    return plan


def run_batched(args):
    print(json.dumps(batched_bench(args)), flush=True)


def batched_bench(args):
    """512 independent filters (zoned / sectorized, sizes log-uniform up to
    2^24) built and probed in one persistent, graph-captured launch vs the
    same work as separate per-filter calls.  Both arms must give the same
    filter words and the same match lists, bit for bit."""
    import ctypes as C

    import torch

    import dtlg
    from dtlg import keygen
    from dtlg.batch import Batch, BatchItem
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    plan = batched_plan(args.batch_filters, max_log2=args.batch_max_log2)
    items = []
    total_words = 0
    filters = []
    for (wb, w, s, z, k), m, n, p in plan:
        f = dtlg.construct(dtlg.blocked_bloomfilter_config(k=k, word_size=wb, word_cnt_per_block=w, sector_cnt=s,
                                                           zone_cnt=z), m)
        filters.append(f)
        total_words += (f.alloc_words() + 3) // 4 * 4  # keep every filter 32-byte aligned
    # all filter words in one allocation, so that one memset resets them per step
    arena = torch.zeros(total_words, dtype=torch.int64, device="cuda")
    off = 0
    n_build = n_probe = 0
    for i, (f, (cfg, m, n, p)) in enumerate(zip(filters, plan)):
        wds = arena[off:off + f.alloc_words()]
        off += (f.alloc_words() + 3) // 4 * 4
        bk = keygen.build_keys_torch(n, 7000 + i)
        pk, _ = keygen.probe_keys_torch(n, p, 0.05, 7000 + i)
        items.append(BatchItem(f, wds, bk, pk, torch.empty(p, dtype=torch.int32, device="cuda"),
                               torch.zeros(1, dtype=torch.int64, device="cuda"), 0))
        n_build += n
        n_probe += p
    stream = torch.cuda.current_stream()
    L = dtlg.lib()
    batch = Batch(items, use_graph=True)
    tuned = batch.autotune(reps=2)   # staging and CTAs per SM, picked by timing

    def batched_step():
        arena.zero_()
        batch.run()

    ws = [torch.empty(L.dtlg_probe_workspace_size(it.probe_keys.numel()), dtype=torch.uint8, device="cuda")
          for it in items]

    def per_filter_step():
        arena.zero_()
        for it, w in zip(items, ws):
            st = L.dtlg_batch_insert(it.filter._h, C.c_void_p(it.filter_data.data_ptr()),
                                     C.c_void_p(it.build_keys.data_ptr()), it.build_keys.numel(), None,
                                     C.c_void_p(stream.cuda_stream))
            assert st == 0, st
            st = L.dtlg_batch_contains_ws(it.filter._h, C.c_void_p(it.filter_data.data_ptr()),
                                          C.c_void_p(it.probe_keys.data_ptr()), it.probe_keys.numel(),
                                          C.c_void_p(it.match_positions.data_ptr()), 0,
                                          C.c_void_p(it.match_cnt.data_ptr()), C.c_void_p(w.data_ptr()),
                                          w.numel(), C.c_void_p(stream.cuda_stream))
            assert st == 0, st

    def timed(fn, steps):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    # results of the two paths must agree bit for bit: every filter's words
    # and every match list
    per_filter_step()
    torch.cuda.synchronize()
    ref_arena = arena.clone()
    ref_counts = [int(it.match_cnt.item()) for it in items]
    ref_lists = [it.match_positions[:c].clone() for it, c in zip(items, ref_counts)]
    for it in items:
        it.match_positions.fill_(-1)
        it.match_cnt.fill_(-1)
    batched_step()
    torch.cuda.synchronize()
    assert torch.equal(arena, ref_arena), "batched filter words differ from the per-filter build"
    for it, c, lst in zip(items, ref_counts, ref_lists):
        assert int(it.match_cnt.item()) == c
        assert torch.equal(it.match_positions[:c], lst)
    del ref_arena, ref_lists
    steps = max(3, min(args.steps, 20))
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    clocks.mark_start()
    ms_batched = timed(batched_step, steps)
    ms_per_filter = timed(per_filter_step, steps)
    clocks.mark_end()
    clk = clocks.stop()
    per_filter_kernels = sum((1 if it.build_keys.numel() else 0) + L.dtlg_probe_kernel_count(it.filter._h,
                                                                                           it.probe_keys.numel())
                             for it in items)
    result = {
        "metric": "batched build+probe of 512 filters: probe Gkeys/s (one persistent graph launch)",
        "value": round(n_probe / (ms_batched / 1e3) / 1e9, 3), "unit": "Gkeys/s", "n_gpus": 1, "steps": steps,
        "warmup": max(3, args.warmup), "ms_per_step": round(ms_batched, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic: seeded u32 bijection keys",
        "config": {"workload": "batched512", "filters": len(items), "build_keys_total": n_build,
                   "probe_keys_total": n_probe, "hit_ratio": 0.05,
                   "filter_configs": [f"u{c[0] * 8} w={c[1]} s={c[2]} z={c[3]} k={c[4]}" for c in BATCH_CONFIGS],
                   "filter_bytes_total": total_words * 8,
                   "step": "zero all filter words, build all filters, probe all filters"},
        "per_filter": {"ms_per_step": round(ms_per_filter, 3), "kernels_per_step": per_filter_kernels + 1,
                       "api": "dtlg_batch_insert + dtlg_batch_contains_ws per filter, one stream"},
        "speedup_vs_per_filter": round(ms_per_filter / ms_batched, 3),
        "gpu_launches": steps * (batch.kernel_count()),
        "fallback_filters": batch.fallback_count(),
        "autotuned": {"staging": tuned["staging"], "ctas_per_sm": tuned["ctas_per_sm"],
                      "staged_filters": batch.staged_count()},
        "bit_exact_vs_per_filter": True,
        "clocks": clk,
    }
    return result


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched512":
        run_batched(args)
    else:
        run_dtlg(args)


if __name__ == "__main__":
    main()
