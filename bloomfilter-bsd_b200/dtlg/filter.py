"""Host-side mirror of the reference's filter API over libdtlg.so.

Mirrors, name for name and argument for argument:
  * dtl::filter::filter_base        (src/dtl/filter/filter_base.hpp:11-62)
  * bbf_32 / bbf_64 / zbbf_32 / zbbf_64 / cf
                                    (src/dtl/filter/{bbf_32,bbf_64,zbbf_32,zbbf_64,cf}.hpp)
  * dtl::blocked_bloomfilter_config (blocked_bloomfilter/blocked_bloomfilter_config.hpp:11-18)
  * dtl::cuckoofilter::config       (cuckoofilter/cuckoofilter_config.hpp:13-16)
  * dtl::filter::filter + probe_t   (src/dtl/filter/filter.hpp:35-261)

Filter words, keys and match positions are CUDA tensors (torch is used only
for device memory and streams); the caller owns the filter words, exactly as
with the reference.  Errors raise: InvalidConfig / SizeError mirror the
reference's std::invalid_argument / std::logic_error.
"""
import ctypes as C
import threading
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib

POWER_OF_TWO = 0   # dtl::block_addressing::POWER_OF_TWO
MAGIC = 1          # dtl::block_addressing::MAGIC


@dataclass
class blocked_bloomfilter_config:  # noqa: N801 (reference name)
    k: int = 8
    word_size: int = 4
    word_cnt_per_block: int = 1
    sector_cnt: int = 1
    addr_mode: int = POWER_OF_TWO
    zone_cnt: int = 1


@dataclass
class cuckoofilter_config:  # noqa: N801 (reference name)
    bits_per_tag: int = 8
    tags_per_bucket: int = 2
    addr_mode: int = POWER_OF_TWO


def _torch():
    import torch
    return torch


def _stream():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev_ptr(t, name):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return C.c_void_p(t.data_ptr())


def as_device_keys(keys, device=None):
    """uint32 keys as a contiguous int32 CUDA tensor (copying host arrays)."""
    torch = _torch()
    if isinstance(keys, torch.Tensor):
        if keys.dtype not in (torch.int32, torch.uint32):
            keys = keys.to(torch.int64).to(torch.int32)
        if not keys.is_cuda:
            keys = keys.to(device or "cuda")
        return keys.contiguous()
    a = np.ascontiguousarray(np.asarray(keys, dtype=np.uint32))
    return torch.from_numpy(a.view(np.int32)).to(device or "cuda")


class filter_base:  # noqa: N801 (reference name)
    """dtl::filter::filter_base (filter_base.hpp:11-62) over libdtlg.so."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                lib().dtlg_destroy(h)
            except Exception:
                pass

    # ---- sizes / name (filter_base.hpp:48-56) ----
    def name(self):
        n = lib().dtlg_name(self._h, None, 0)
        buf = C.create_string_buffer(n + 1)
        lib().dtlg_name(self._h, buf, n + 1)
        return buf.value.decode()

    def size_in_bytes(self):
        return lib().dtlg_size_in_bytes(self._h)

    def size(self):
        """Filter size in 64-bit words (filter_base.hpp:54-56)."""
        return lib().dtlg_size(self._h)

    def alloc_words(self):
        """64-bit words to allocate: size() plus, for cuckoo, the victim record."""
        return lib().dtlg_alloc_words_u64(self._h)

    def block_cnt(self):
        return lib().dtlg_block_cnt(self._h)

    def is_magic(self):
        return bool(lib().dtlg_is_magic(self._h))

    def kind(self):
        return ("bloom", "zoned", "cuckoo", "blocked_cuckoo", "classic_bloom")[lib().dtlg_kind(self._h)]

    def set_probe_options(self, mode=0, variant=-1):
        """Probe kernel choice (0 auto, 1 fused, 2 bitmask + compaction) and the
        bitmask kernel's register budget; results are identical in all modes."""
        check(lib().dtlg_set_probe_options(self._h, int(mode), int(variant)), "set_probe_options")

    def set_probe_passes(self, passes=0):
        """Block-range passes of the two-kernel probe (0 = automatic)."""
        check(lib().dtlg_set_probe_passes(self._h, int(passes)), "set_probe_passes")

    def set_build_options(self, mode=0):
        """Bloom build plan: 0 automatic, 1 one kernel of global atomic ORs,
        2 keys grouped by L2-sized block range first (same words)."""
        check(lib().dtlg_set_build_options(self._h, int(mode)), "set_build_options")

    def autotune(self, filter_data, keys, reps=5):
        """Times every probe plan on these keys and keeps the fastest for this
        filter (the reference's calibrate(), blocked_bloomfilter_tune_impl.hpp:
        162-268); returns {"mode", "variant", "passes", "ms", "gkeys_per_s"}."""
        torch = _torch()
        keys = as_device_keys(keys, filter_data.device)
        pos = torch.empty(max(1, keys.numel()), dtype=torch.int32, device=keys.device)
        plan = _lib.ProbePlanS()
        check(lib().dtlg_autotune_probe(self._h, _dev_ptr(filter_data, "filter_data"), _dev_ptr(keys, "keys"),
                                        keys.numel(), _dev_ptr(pos, "match_positions"), int(reps), _stream(),
                                        C.byref(plan)), "autotune_probe")
        return {"mode": plan.mode, "variant": plan.variant, "passes": plan.passes, "ms": plan.ms,
                "gkeys_per_s": plan.gkeys_per_s}

    def alloc_filter_data(self, device="cuda"):
        """Zeroed filter words, as the facade allocates them (filter.hpp:113-119)."""
        torch = _torch()
        return torch.zeros(max(1, self.alloc_words()), dtype=torch.int64, device=device)

    # ---- API (filter_base.hpp:20-45) ----
    def insert(self, filter_data, key):
        st = lib().dtlg_insert(self._h, _dev_ptr(filter_data, "filter_data"), int(key) & 0xFFFFFFFF, _stream())
        if st == 7:
            return False
        check(st, "insert")
        return True

    def batch_insert(self, filter_data, keys, key_cnt=None):
        """Returns False when a cuckoo key could not be placed (the reference's
        result, cuckoofilter_logic.hpp:330-337); Bloom inserts never fail."""
        keys = as_device_keys(keys, filter_data.device)
        n = keys.numel() if key_cnt is None else int(key_cnt)
        failed = C.c_uint64(0)
        st = lib().dtlg_batch_insert(self._h, _dev_ptr(filter_data, "filter_data"), _dev_ptr(keys, "keys"), n,
                                     C.byref(failed), _stream())
        self.last_failed = failed.value
        if st == 7:
            return False
        check(st, "batch_insert")
        return True

    def contains(self, filter_data, key):
        r = C.c_int(0)
        check(lib().dtlg_contains(self._h, _dev_ptr(filter_data, "filter_data"), int(key) & 0xFFFFFFFF,
                                  C.byref(r), _stream()), "contains")
        return bool(r.value)

    def batch_contains(self, filter_data, keys, key_cnt, match_positions, match_offset=0):
        """Writes the ascending positions i + match_offset of matching keys to
        match_positions (capacity >= key_cnt); returns the match count."""
        cnt = C.c_uint64(0)
        check(lib().dtlg_batch_contains(self._h, _dev_ptr(filter_data, "filter_data"), _dev_ptr(keys, "keys"),
                                        int(key_cnt), _dev_ptr(match_positions, "match_positions"),
                                        int(match_offset) & 0xFFFFFFFF, C.byref(cnt), _stream()),
              "batch_contains")
        return cnt.value

    def batch_contains_async(self, filter_data, keys, key_cnt, match_positions, match_offset, match_cnt_dev):
        check(lib().dtlg_batch_contains_async(self._h, _dev_ptr(filter_data, "filter_data"),
                                              _dev_ptr(keys, "keys"), int(key_cnt),
                                              _dev_ptr(match_positions, "match_positions"),
                                              int(match_offset) & 0xFFFFFFFF, _dev_ptr(match_cnt_dev, "count"),
                                              _stream()), "batch_contains_async")

    def batch_contains_gather(self, filter_data, keys, cols, out_cols, match_positions=None, match_offset=0):
        """batch_contains fused with the gather of the matching rows of payload
        columns (CUDA tensors of 4- or 8-byte elements, one row per key):
        out_cols[c][j] = cols[c][i] for the j-th match i.  Returns the count."""
        torch = _torch()
        keys = as_device_keys(keys, filter_data.device)
        n = keys.numel()
        if len(cols) != len(out_cols) or len(cols) > 4:
            raise ValueError("up to 4 payload columns, one output column each")
        cp = (C.c_void_p * max(1, len(cols)))(*[_dev_ptr(c, "cols").value for c in cols])
        op = (C.c_void_p * max(1, len(cols)))(*[_dev_ptr(o, "out_cols").value for o in out_cols])
        cb = (C.c_uint32 * max(1, len(cols)))(*[c.element_size() for c in cols])
        for c, o in zip(cols, out_cols):
            if c.numel() < n or o.numel() < n or c.element_size() != o.element_size():
                raise ValueError("payload columns need one row per key and outputs of the same type")
        ws = torch.empty(lib().dtlg_probe_workspace_size(n), dtype=torch.uint8, device=filter_data.device)
        cnt = torch.zeros(1, dtype=torch.int64, device=filter_data.device)
        check(lib().dtlg_batch_contains_gather(self._h, _dev_ptr(filter_data, "filter_data"), _dev_ptr(keys, "keys"),
                                               n, len(cols), cp, cb, op,
                                               _dev_ptr(match_positions, "match_positions")
                                               if match_positions is not None else None,
                                               int(match_offset) & 0xFFFFFFFF, _dev_ptr(cnt, "count"),
                                               _dev_ptr(ws, "workspace"), ws.numel(), _stream()),
              "batch_contains_gather")
        return int(cnt.item())

    def batch_contains_host(self, filter_data, keys_host, match_positions_host, match_offset=0):
        """Host key / position buffers (numpy uint32), device filter words."""
        keys_host = np.ascontiguousarray(keys_host, dtype=np.uint32)
        assert match_positions_host.dtype == np.uint32 and match_positions_host.size >= keys_host.size
        cnt = C.c_uint64(0)
        check(lib().dtlg_batch_contains_host(self._h, _dev_ptr(filter_data, "filter_data"),
                                             C.c_void_p(keys_host.ctypes.data), keys_host.size,
                                             C.c_void_p(match_positions_host.ctypes.data),
                                             int(match_offset) & 0xFFFFFFFF, C.byref(cnt), _stream()),
              "batch_contains_host")
        return cnt.value

    def batch_insert_host(self, filter_data, keys_host):
        keys_host = np.ascontiguousarray(keys_host, dtype=np.uint32)
        failed = C.c_uint64(0)
        st = lib().dtlg_batch_insert_host(self._h, _dev_ptr(filter_data, "filter_data"),
                                          C.c_void_p(keys_host.ctypes.data), keys_host.size, C.byref(failed),
                                          _stream())
        self.last_failed = failed.value
        if st == 7:
            return False
        check(st, "batch_insert_host")
        return True


def set_l2_fetch_granularity(nbytes):
    """cudaLimitMaxL2FetchGranularity of the current device's context (this
    process only); returns the value in effect."""
    v = C.c_int(0)
    check(lib().dtlg_set_l2_fetch_granularity(int(nbytes), C.byref(v)), "set_l2_fetch_granularity")
    return v.value


def _bloom_handle(m, k, word_size, w, s, z):
    cfg = _lib.BloomConfigS(k, word_size, w, s, 0, z)
    h = C.c_void_p()
    check(lib().dtlg_bloom_create(C.byref(cfg), int(m), C.byref(h)),
          f"blocked Bloom filter k={k}, word_size={word_size}, w={w}, s={s}, z={z}")
    return h


class bbf_32(filter_base):  # noqa: N801 -- bbf_32.hpp:53
    def __init__(self, m, k, word_cnt_per_block=1, sector_cnt=1):
        super().__init__(_bloom_handle(m, k, 4, word_cnt_per_block, sector_cnt, 1))


class bbf_64(filter_base):  # noqa: N801 -- bbf_64.hpp
    def __init__(self, m, k, word_cnt_per_block=1, sector_cnt=1):
        super().__init__(_bloom_handle(m, k, 8, word_cnt_per_block, sector_cnt, 1))


class zbbf_32(filter_base):  # noqa: N801 -- zbbf_32.hpp
    def __init__(self, m, k, word_cnt_per_block=4, zone_cnt=2):
        super().__init__(_bloom_handle(m, k, 4, word_cnt_per_block, word_cnt_per_block, zone_cnt))


class zbbf_64(filter_base):  # noqa: N801 -- zbbf_64.hpp
    def __init__(self, m, k, word_cnt_per_block=4, zone_cnt=2):
        super().__init__(_bloom_handle(m, k, 8, word_cnt_per_block, word_cnt_per_block, zone_cnt))


class cf(filter_base):  # noqa: N801 -- cf.hpp, cf.cpp:18,27
    def __init__(self, m, bits_per_tag=16, tags_per_bucket=4):
        cfg = _lib.CuckooConfigS(bits_per_tag, tags_per_bucket, 0)
        h = C.c_void_p()
        check(lib().dtlg_cuckoo_create(C.byref(cfg), int(m), C.byref(h)),
              f"cuckoo filter t={bits_per_tag}, b={tags_per_bucket}")
        super().__init__(h)
        self.bits_per_tag, self.tags_per_bucket = bits_per_tag, tags_per_bucket

    def count_occupied_slots(self, filter_data):
        c = C.c_uint64(0)
        check(lib().dtlg_count_occupied_slots(self._h, _dev_ptr(filter_data, "filter_data"), C.byref(c),
                                              _stream()), "count_occupied_slots")
        return c.value

    def get_bucket_count(self):
        return self.block_cnt()


class bcf(filter_base):  # noqa: N801 -- bcf.hpp:56, bcf.cpp:24-25
    """The blocked cuckoo filter dtl::bcf: blocks of block_size_bytes, each a
    small cuckoo table of one-word buckets.  Inserts never fail (bcf.cpp:36-40).
    Unlike the reference's bcf::size() (32-bit words), size() here counts
    64-bit words, like every filter_base."""

    def __init__(self, m, block_size_bytes=64, tag_size_bits=16, associativity=4):
        cfg = _lib.BcfConfigS(block_size_bytes, tag_size_bits, associativity)
        h = C.c_void_p()
        check(lib().dtlg_blocked_cuckoo_create(C.byref(cfg), int(m), C.byref(h)),
              f"blocked cuckoo filter block={block_size_bytes}, t={tag_size_bits}, a={associativity}")
        super().__init__(h)
        self.block_size_bytes = block_size_bytes
        self.tag_size_bits, self.associativity = tag_size_bits, associativity


class bloomfilter_logic(filter_base):  # noqa: N801 -- bloomfilter/bloomfilter_logic.hpp:22-64
    """The classic Bloom filter: one bit in each of k independently addressed
    32-bit words, k <= 17.  The addressing is the reference's template
    argument (POWER_OF_TWO or MAGIC), not derived from m."""

    def __init__(self, m, k, addressing=None):
        addressing = POWER_OF_TWO if addressing is None else addressing
        cfg = _lib.ClassicConfigS(k, 1 if addressing == MAGIC else 0)
        h = C.c_void_p()
        check(lib().dtlg_classic_bloom_create(C.byref(cfg), int(m), C.byref(h)), f"classic Bloom filter k={k}")
        super().__init__(h)
        self.k = k


def construct(config, m):
    """filter.hpp:42-72: the filter for a config (word size 4/8, zone_cnt 1 =
    blocked or sectorized, > 1 = zoned; cuckoo by cuckoofilter_config)."""
    if isinstance(config, cuckoofilter_config):
        return cf(m, config.bits_per_tag, config.tags_per_bucket)
    if config.word_size == 4:
        if config.zone_cnt == 1:
            return bbf_32(m, config.k, config.word_cnt_per_block, config.sector_cnt)
        return zbbf_32(m, config.k, config.word_cnt_per_block, config.zone_cnt)
    if config.word_size == 8:
        if config.zone_cnt == 1:
            return bbf_64(m, config.k, config.word_cnt_per_block, config.sector_cnt)
        return zbbf_64(m, config.k, config.word_cnt_per_block, config.zone_cnt)
    raise _lib.InvalidConfig(1, "Illegal configuration. Word size must be either 4 or 8.")


class DeviceReplicas:
    """The filter words once per device, each copy made on first use.

    The GPU counterpart of the reference's per-NUMA-node replicas
    (filter.hpp:98-101,128-152): the words live on the device that built them
    (`home`); the first probe from another device copies them there, under a
    lock with a second check, as the reference does per memory node.  `copy`
    makes one replica: copy(home_words, device) -> words on that device.  An
    insert makes every replica stale, so invalidate() drops them (the
    reference leaves inserting after probing undefined, filter.hpp:33-34).
    """

    def __init__(self, words, home, copy):
        self.home = home
        self._words = {home: words}
        self._copy = copy
        self._lock = threading.Lock()

    def get(self, device):
        w = self._words.get(device)
        if w is not None:
            return w
        with self._lock:
            w = self._words.get(device)
            if w is None:                      # double check, as filter.hpp:139-147
                w = self._copy(self._words[self.home], device)
                self._words[device] = w
        return w

    def devices(self):
        return sorted(self._words)

    def invalidate(self):
        with self._lock:
            self._words = {self.home: self._words[self.home]}


def _peer_replica(words, device):
    """A copy of the filter words on `device`: a copy-engine transfer
    (dtlg_copy_words_peer), no kernel reads the other device's memory."""
    torch = _torch()
    dst = torch.empty(words.numel(), dtype=words.dtype, device=torch.device("cuda", device))
    with torch.cuda.device(device):
        st = lib().dtlg_copy_words_peer(C.c_void_p(dst.data_ptr()), device, C.c_void_p(words.data_ptr()),
                                        words.device.index, words.numel(), _stream())
        check(st, "dtlg_copy_words_peer")
        torch.cuda.current_stream().synchronize()
    return dst


class filter:  # noqa: N801 -- dtl::filter::filter (filter.hpp:35-261)
    """Construct by config, insert, then probe through probe instances.

    As in the reference, insert() must not be called after probe() handed out
    a probe instance (filter.hpp:33-34); here it drops the replicas.  The
    words are built on one CUDA device and replicated to every other device
    that probes them (DeviceReplicas).
    """

    def __init__(self, config, m, device="cuda"):
        self.filter_instance = construct(config, m)
        self.filter_data = self.filter_instance.alloc_filter_data(device)
        self.replicas = DeviceReplicas(self.filter_data, self.filter_data.device.index, _peer_replica)

    @staticmethod
    def for_workload(n, work_ns, fpr_target=0.1, hit_ratio=0.0, l2_resident=False, method="mlp", device="cuda"):
        """The filter the cost model picks for n build keys and work_ns of
        downstream work per passing tuple -- construct(n, tw, ...) of the
        reference (filter.hpp:76-82), which reads its skyline matrix.  method:
        "mlp" (the trained network, GPU), "skyline" (the reference's cached
        lookup) or "exhaustive" (the calibrated search)."""
        from .model.planner import shared_planner
        cfg, m = shared_planner().config_for(n, fpr_target, hit_ratio, work_ns, l2_resident, method)
        return filter(cfg, m, device)

    def insert(self, keys):
        torch = _torch()
        self.replicas.invalidate()
        with torch.cuda.device(self.filter_data.device):
            if isinstance(keys, torch.Tensor) and keys.is_cuda:
                keys = keys.to(self.filter_data.device)
                return self.filter_instance.batch_insert(self.filter_data, keys)
            return self.filter_instance.batch_insert_host(self.filter_data, np.asarray(keys, dtype=np.uint32))

    def filter_data_on(self, device):
        """The words on `device` (an index), replicated there on first use
        (filter_shared::get_filter_data_ptr, filter.hpp:128-152)."""
        return self.replicas.get(device)

    def probe(self):
        return probe_t(self)


class probe_t:  # noqa: N801 -- filter.hpp:205-253
    """Probes against the replica on the device of the keys (host keys: the
    current device).  The reference's probe_t fetches its node's replica
    (filter.hpp:212-215) but then probes the original words
    (filter.hpp:234-240); here the replica is the one probed."""

    def __init__(self, f):
        self._f = f

    def device_of(self, keys):
        torch = _torch()
        if isinstance(keys, torch.Tensor) and keys.is_cuda:
            return keys.device.index
        return torch.cuda.current_device()

    def __call__(self, keys, match_pos=None, match_offset=0):
        """Returns the match count; positions go to match_pos (a CUDA tensor
        for device keys, a numpy uint32 array for host keys)."""
        torch = _torch()
        dev = self.device_of(keys)
        fi, data = self._f.filter_instance, self._f.filter_data_on(dev)
        with torch.cuda.device(dev):
            if isinstance(keys, torch.Tensor) and keys.is_cuda:
                if match_pos is None:
                    match_pos = torch.empty(max(1, keys.numel()), dtype=torch.int32, device=keys.device)
                return fi.batch_contains(data, keys.contiguous(), keys.numel(), match_pos, match_offset)
            keys = np.ascontiguousarray(keys, dtype=np.uint32)
            if match_pos is None:
                match_pos = np.empty(max(1, keys.size), dtype=np.uint32)
            return fi.batch_contains_host(data, keys, match_pos, match_offset)
