"""ctypes bindings of the test oracles.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline / reference legs, never by the product package.

* ``Bloom`` / ``Cuckoo`` / ``BlockedCuckoo`` / ``ClassicBloom`` wrap
  liboracle.so, the C restatement (dtl_oracle.c).
* ``RefLib`` wraps oracle/_ref/libdtlref_*.so, the reference's own filter logic
  compiled from its sources (see oracle/Makefile); absent when not built.
  ``RefBcf`` wraps oracle/_ref/libdtlref_bcf*.so, the reference's dtl::bcf;
  ``RefCbf`` oracle/_ref/libdtlref_cbf.so, its classic Bloom filter.
"""
import ctypes as C
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


class _Addr(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("block_cnt", C.c_uint32), ("block_cnt_log2", C.c_uint32),
                ("block_cnt_mask", C.c_uint32), ("magic", C.c_uint32), ("shift", C.c_uint32)]


class _BloomS(C.Structure):
    _fields_ = [("word_bytes", C.c_uint32), ("w", C.c_uint32), ("s", C.c_uint32), ("z", C.c_uint32),
                ("k", C.c_uint32), ("addr", _Addr), ("m", C.c_uint64), ("m_actual", C.c_uint64),
                ("word_cnt", C.c_uint64), ("size_u64", C.c_uint64)]


class _CuckooS(C.Structure):
    _fields_ = [("t", C.c_uint32), ("b", C.c_uint32), ("bytes_per_bucket", C.c_uint32), ("addr", _Addr),
                ("m", C.c_uint64), ("m_actual", C.c_uint64), ("table_words_u32", C.c_uint64),
                ("size_u64", C.c_uint64), ("alloc_u64", C.c_uint64)]


class _BcfS(C.Structure):
    _fields_ = [("block_bytes", C.c_uint32), ("t", C.c_uint32), ("a", C.c_uint32), ("word_bytes", C.c_uint32),
                ("bucket_bits", C.c_uint32), ("hash_shift", C.c_uint32), ("addr", _Addr), ("m", C.c_uint64),
                ("m_actual", C.c_uint64), ("word_cnt", C.c_uint64), ("size_u32", C.c_uint64)]


class _CbfS(C.Structure):
    _fields_ = [("k", C.c_uint32), ("addr", _Addr), ("bit_shift", C.c_uint32), ("bit_mask", C.c_uint32),
                ("m", C.c_uint64), ("m_actual", C.c_uint64), ("word_cnt", C.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle)")
        L = C.CDLL(path)
        L.orc_hash.restype = C.c_uint32
        L.orc_hash.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_next_cheap_magic.restype = C.c_int
        L.orc_next_cheap_magic.argtypes = [C.c_uint32] + [C.POINTER(C.c_uint32)] * 3
        L.orc_fast_mod.restype = C.c_uint32
        L.orc_fast_mod.argtypes = [C.c_uint32] * 4
        L.orc_bloom_init.restype = C.c_int
        L.orc_bloom_init.argtypes = [C.POINTER(_BloomS)] + [C.c_uint32] * 5 + [C.c_uint64]
        L.orc_bloom_insert.argtypes = [C.POINTER(_BloomS), C.c_void_p, _u32p, C.c_uint64, C.c_int]
        L.orc_bloom_contains.restype = C.c_int
        L.orc_bloom_contains.argtypes = [C.POINTER(_BloomS), C.c_void_p, C.c_uint32, C.c_int]
        L.orc_bloom_batch_contains.restype = C.c_uint64
        L.orc_bloom_batch_contains.argtypes = [C.POINTER(_BloomS), C.c_void_p, _u32p, C.c_uint32,
                                               _u32p, C.c_uint32, C.c_int]
        L.orc_bloom_batch_contains_mt.restype = C.c_uint64
        L.orc_bloom_batch_contains_mt.argtypes = [C.POINTER(_BloomS), C.c_void_p, _u32p, C.c_uint64,
                                                  _u32p, C.c_int]
        L.orc_bloom_bits.argtypes = [C.POINTER(_BloomS), C.c_uint32, C.c_int, _u32p, _u32p]
        L.orc_cuckoo_init.restype = C.c_int
        L.orc_cuckoo_init.argtypes = [C.POINTER(_CuckooS), C.c_uint32, C.c_uint32, C.c_uint64]
        L.orc_cuckoo_insert.restype = C.c_int
        L.orc_cuckoo_insert.argtypes = [C.POINTER(_CuckooS), C.c_void_p, _u32p, C.c_uint64, C.c_uint64]
        L.orc_cuckoo_contains.restype = C.c_int
        L.orc_cuckoo_contains.argtypes = [C.POINTER(_CuckooS), C.c_void_p, C.c_uint32]
        L.orc_cuckoo_batch_contains.restype = C.c_uint64
        L.orc_cuckoo_batch_contains.argtypes = [C.POINTER(_CuckooS), C.c_void_p, _u32p, C.c_uint32,
                                                _u32p, C.c_uint32]
        L.orc_cuckoo_count_occupied.restype = C.c_uint64
        L.orc_cuckoo_count_occupied.argtypes = [C.POINTER(_CuckooS), C.c_void_p]
        L.orc_cuckoo_read_tag.restype = C.c_uint32
        L.orc_cuckoo_read_tag.argtypes = [C.POINTER(_CuckooS), C.c_void_p, C.c_uint64, C.c_uint32]
        L.orc_cuckoo_index_tag.argtypes = [C.POINTER(_CuckooS), C.c_uint32] + [C.POINTER(C.c_uint32)] * 3
        L.orc_bcf_init.restype = C.c_int
        L.orc_bcf_init.argtypes = [C.POINTER(_BcfS)] + [C.c_uint32] * 3 + [C.c_uint64]
        L.orc_bcf_insert.argtypes = [C.POINTER(_BcfS), C.c_void_p, _u32p, C.c_uint64, C.c_uint64]
        L.orc_bcf_contains.restype = C.c_int
        L.orc_bcf_contains.argtypes = [C.POINTER(_BcfS), C.c_void_p, C.c_uint32]
        L.orc_bcf_batch_contains.restype = C.c_uint64
        L.orc_bcf_batch_contains.argtypes = [C.POINTER(_BcfS), C.c_void_p, _u32p, C.c_uint32, _u32p, C.c_uint32]
        L.orc_bcf_locate.argtypes = [C.POINTER(_BcfS), C.c_uint32] + [C.POINTER(C.c_uint32)] * 4
        L.orc_cbf_init.restype = C.c_int
        L.orc_cbf_init.argtypes = [C.POINTER(_CbfS), C.c_uint32, C.c_uint64, C.c_uint32]
        L.orc_cbf_insert.argtypes = [C.POINTER(_CbfS), C.c_void_p, _u32p, C.c_uint64]
        L.orc_cbf_contains.restype = C.c_int
        L.orc_cbf_contains.argtypes = [C.POINTER(_CbfS), C.c_void_p, C.c_uint32]
        L.orc_cbf_batch_contains.restype = C.c_uint64
        L.orc_cbf_batch_contains.argtypes = [C.POINTER(_CbfS), C.c_void_p, _u32p, C.c_uint32, _u32p, C.c_uint32]
        _lib = L
    return _lib


def _keys(keys):
    return np.ascontiguousarray(keys, dtype=np.uint32)


def next_cheap_magic(n):
    d, mg, sh = C.c_uint32(), C.c_uint32(), C.c_uint32()
    if not lib().orc_next_cheap_magic(n, C.byref(d), C.byref(mg), C.byref(sh)):
        raise ValueError("no cheap magic divisor")
    return d.value, mg.value, sh.value


class Bloom:
    """C restatement of one blocked Bloom filter config (data owned by caller)."""

    def __init__(self, word_bytes, w, s, z, k, m):
        self.s_ = _BloomS()
        rc = lib().orc_bloom_init(C.byref(self.s_), word_bytes, w, s, z, k, m)
        if rc:
            raise ValueError(f"invalid bloom config rc={rc}")

    @property
    def size_u64(self):
        return self.s_.size_u64

    @property
    def word_cnt(self):
        return self.s_.word_cnt

    @property
    def m_actual(self):
        return self.s_.m_actual

    @property
    def block_cnt(self):
        return self.s_.addr.block_cnt

    @property
    def magic(self):
        return self.s_.addr.mode == 1

    def alloc(self):
        return np.zeros(max(1, self.size_u64), dtype=np.uint64)

    def insert(self, data, keys, stale_k8=True):
        k = _keys(keys)
        lib().orc_bloom_insert(C.byref(self.s_), data.ctypes.data, k, len(k), int(stale_k8))

    def contains(self, data, key, stale_k8=True):
        return bool(lib().orc_bloom_contains(C.byref(self.s_), data.ctypes.data, int(key), int(stale_k8)))

    def batch_contains(self, data, keys, match_offset=0, stale_k8=True):
        k = _keys(keys)
        out = np.zeros(max(1, len(k)), dtype=np.uint32)
        n = lib().orc_bloom_batch_contains(C.byref(self.s_), data.ctypes.data, k, len(k), out,
                                           match_offset & 0xFFFFFFFF, int(stale_k8))
        return out[:n].copy()

    def batch_contains_mt(self, data, keys, threads):
        k = _keys(keys)
        out = np.zeros(max(1, len(k)), dtype=np.uint32)
        return lib().orc_bloom_batch_contains_mt(C.byref(self.s_), data.ctypes.data, k, len(k), out,
                                                 threads)

    def bits(self, key, stale_k8=True):
        wi = np.zeros(16, dtype=np.uint32)
        bi = np.zeros(16, dtype=np.uint32)
        lib().orc_bloom_bits(C.byref(self.s_), int(key), int(stale_k8), wi, bi)
        return wi[: self.s_.k].copy(), bi[: self.s_.k].copy()


class Cuckoo:
    """C restatement of one cuckoo filter config (data owned by caller)."""

    def __init__(self, t, b, m):
        self.s_ = _CuckooS()
        rc = lib().orc_cuckoo_init(C.byref(self.s_), t, b, m)
        if rc:
            raise ValueError(f"invalid cuckoo config rc={rc}")

    @property
    def alloc_u64(self):
        return self.s_.alloc_u64

    @property
    def size_u64(self):
        return self.s_.size_u64

    @property
    def bucket_cnt(self):
        return self.s_.addr.block_cnt

    @property
    def table_words_u32(self):
        return self.s_.table_words_u32

    def alloc(self):
        return np.zeros(self.alloc_u64, dtype=np.uint64)

    def insert(self, data, keys, seed=1):
        k = _keys(keys)
        return bool(lib().orc_cuckoo_insert(C.byref(self.s_), data.ctypes.data, k, len(k), seed))

    def contains(self, data, key):
        return bool(lib().orc_cuckoo_contains(C.byref(self.s_), data.ctypes.data, int(key)))

    def batch_contains(self, data, keys, match_offset=0):
        k = _keys(keys)
        out = np.zeros(max(1, len(k)), dtype=np.uint32)
        n = lib().orc_cuckoo_batch_contains(C.byref(self.s_), data.ctypes.data, k, len(k), out,
                                            match_offset & 0xFFFFFFFF)
        return out[:n].copy()

    def count_occupied(self, data):
        return lib().orc_cuckoo_count_occupied(C.byref(self.s_), data.ctypes.data)

    def index_tag(self, key):
        a, b, t = C.c_uint32(), C.c_uint32(), C.c_uint32()
        lib().orc_cuckoo_index_tag(C.byref(self.s_), int(key), C.byref(a), C.byref(b), C.byref(t))
        return a.value, b.value, t.value


class BlockedCuckoo:
    """C restatement of one blocked cuckoo filter config (data owned by caller)."""

    def __init__(self, m, block_bytes=64, t=16, a=4):
        self.s_ = _BcfS()
        rc = lib().orc_bcf_init(C.byref(self.s_), block_bytes, t, a, m)
        if rc:
            raise ValueError(f"invalid blocked cuckoo config rc={rc}")

    @property
    def size_u32(self):
        return self.s_.size_u32

    @property
    def size_u64(self):
        return (self.s_.size_u32 + 1) // 2

    @property
    def m_actual(self):
        return self.s_.m_actual

    @property
    def block_cnt(self):
        return self.s_.addr.block_cnt

    @property
    def magic(self):
        return self.s_.addr.mode == 1

    @property
    def word_bytes(self):
        return self.s_.word_bytes

    @property
    def hash_shift(self):
        return self.s_.hash_shift

    def alloc(self):
        return np.zeros(max(1, self.size_u64), dtype=np.uint64)

    def insert(self, data, keys, seed=1):
        k = _keys(keys)
        lib().orc_bcf_insert(C.byref(self.s_), data.ctypes.data, k, len(k), seed)

    def contains(self, data, key):
        return bool(lib().orc_bcf_contains(C.byref(self.s_), data.ctypes.data, int(key)))

    def batch_contains(self, data, keys, match_offset=0):
        k = _keys(keys)
        out = np.zeros(max(1, len(k)), dtype=np.uint32)
        n = lib().orc_bcf_batch_contains(C.byref(self.s_), data.ctypes.data, k, len(k), out,
                                         match_offset & 0xFFFFFFFF)
        return out[:n].copy()

    def locate(self, key):
        r = [C.c_uint32() for _ in range(4)]
        lib().orc_bcf_locate(C.byref(self.s_), int(key), *[C.byref(x) for x in r])
        return tuple(x.value for x in r)  # block, bucket 1, bucket 2, tag


class ClassicBloom:
    """C restatement of the classic Bloom filter (data owned by caller)."""

    def __init__(self, k, m, magic=False):
        self.s_ = _CbfS()
        rc = lib().orc_cbf_init(C.byref(self.s_), k, m, 1 if magic else 0)
        if rc:
            raise ValueError(f"invalid classic Bloom config rc={rc}")

    @property
    def word_cnt(self):
        return self.s_.word_cnt

    @property
    def m_actual(self):
        return self.s_.m_actual

    @property
    def block_cnt(self):
        return self.s_.addr.block_cnt

    def alloc(self):
        return np.zeros(max(1, (self.word_cnt + 1) // 2), dtype=np.uint64)

    def insert(self, data, keys):
        k = _keys(keys)
        lib().orc_cbf_insert(C.byref(self.s_), data.ctypes.data, k, len(k))

    def contains(self, data, key):
        return bool(lib().orc_cbf_contains(C.byref(self.s_), data.ctypes.data, int(key)))

    def batch_contains(self, data, keys, match_offset=0):
        k = _keys(keys)
        out = np.zeros(max(1, len(k)), dtype=np.uint32)
        n = lib().orc_cbf_batch_contains(C.byref(self.s_), data.ctypes.data, k, len(k), out,
                                         match_offset & 0xFFFFFFFF)
        return out[:n].copy()


# --------------------------------------------------------------------------
# The reference compiled from its sources (oracle/_ref)
# --------------------------------------------------------------------------
def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


class RefLib:
    """The reference's filter logic (oracle/_ref/libdtlref_{avx512,avx2}.so)."""

    def __init__(self, variant=None):
        flags = _cpu_flags()
        if variant is None:
            variant = "avx512" if {"avx512f", "avx512bw", "avx512dq", "avx512vl"} <= flags else "avx2"
        path = os.path.join(HERE, "_ref", f"libdtlref_{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.variant = variant
        self.path = path
        L = C.CDLL(path)
        vp = C.c_void_p
        L.ref_simd_lanes.restype = C.c_int
        L.ref_bloom_create.restype = vp
        L.ref_bloom_create.argtypes = [C.c_uint32] * 5 + [C.c_uint64]
        L.ref_cuckoo_create.restype = vp
        L.ref_cuckoo_create.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64]
        L.ref_instance_count.restype = C.c_int
        L.ref_instance_count.argtypes = [C.c_int]
        L.ref_destroy.argtypes = [vp]
        L.ref_word_cnt.restype = C.c_uint64
        L.ref_word_cnt.argtypes = [vp]
        L.ref_length.restype = C.c_uint64
        L.ref_length.argtypes = [vp]
        L.ref_insert.restype = C.c_int
        L.ref_insert.argtypes = [vp, vp, _u32p, C.c_uint32]
        L.ref_contains.restype = C.c_int
        L.ref_contains.argtypes = [vp, vp, C.c_uint32]
        L.ref_batch_contains.restype = C.c_uint64
        L.ref_batch_contains.argtypes = [vp, vp, _u32p, C.c_uint32, _u32p, C.c_uint32, C.c_int]
        L.ref_count_occupied.restype = C.c_uint64
        L.ref_count_occupied.argtypes = [vp, vp]
        L.ref_batch_contains_mt.restype = C.c_uint64
        L.ref_batch_contains_mt.argtypes = [vp, vp, _u32p, C.c_uint64, _u32p, C.c_int, C.c_int]
        L.ref_insert_mt.argtypes = [vp, vp, _u32p, C.c_uint64, C.c_int]
        L.ref_batch_contains_mt_list.restype = C.c_uint64
        L.ref_batch_contains_mt_list.argtypes = [vp, vp, _u32p, C.c_uint64, _u32p, C.c_int, C.c_int]
        L.ref_next_cheap_magic.restype = C.c_int
        L.ref_next_cheap_magic.argtypes = [C.c_uint32] + [C.POINTER(C.c_uint32)] * 3
        self.L = L
        self.lanes = L.ref_simd_lanes()

    def bloom(self, word_bytes, w, s, z, k, m):
        h = self.L.ref_bloom_create(word_bytes, w, s, z, k, m)
        return _RefFilter(self, h) if h else None

    def next_cheap_magic(self, n):
        d, mg, sh = C.c_uint32(), C.c_uint32(), C.c_uint32()
        if not self.L.ref_next_cheap_magic(n, C.byref(d), C.byref(mg), C.byref(sh)):
            raise ValueError("no cheap magic divisor")
        return d.value, mg.value, sh.value

    def cuckoo(self, t, b, m):
        h = self.L.ref_cuckoo_create(t, b, m)
        return _RefFilter(self, h) if h else None


class _RefFilter:
    def __init__(self, ref, h):
        self.ref, self.h = ref, h

    def __del__(self):
        try:
            self.ref.L.ref_destroy(self.h)
        except Exception:
            pass

    @property
    def word_cnt(self):
        return self.ref.L.ref_word_cnt(self.h)

    @property
    def length(self):
        return self.ref.L.ref_length(self.h)

    def insert(self, data, keys):
        k = _keys(keys)
        return bool(self.ref.L.ref_insert(self.h, data.ctypes.data, k, len(k)))

    def insert_mt(self, data, keys, threads):
        k = _keys(keys)
        self.ref.L.ref_insert_mt(self.h, data.ctypes.data, k, len(k), threads)

    def contains(self, data, key):
        return bool(self.ref.L.ref_contains(self.h, data.ctypes.data, int(key)))

    def batch_contains(self, data, keys, match_offset=0, unroll=1):
        k = _keys(keys)
        out = np.zeros(len(k) + 16, dtype=np.uint32)
        n = self.ref.L.ref_batch_contains(self.h, data.ctypes.data, k, len(k), out,
                                          match_offset & 0xFFFFFFFF, unroll)
        return out[:n].copy()

    def batch_contains_mt(self, data, keys, threads, unroll=1, out=None):
        k = _keys(keys)
        if out is None:
            out = np.zeros(len(k) + 16, dtype=np.uint32)
        return self.ref.L.ref_batch_contains_mt(self.h, data.ctypes.data, k, len(k), out, threads, unroll)

    def batch_contains_mt_list(self, data, keys, threads, unroll=1, out=None):
        """All host threads, each on its own contiguous slice in 1024-key
        batches, then the slices' lists joined: the ascending positions
        (match_offset 0) of every matching key.  Returns a view of `out`."""
        k = _keys(keys)
        if out is None:
            out = np.zeros(len(k) + 64, dtype=np.uint32)
        n = self.ref.L.ref_batch_contains_mt_list(self.h, data.ctypes.data, k, len(k), out, threads, unroll)
        return out[:n]

    def count_occupied(self, data):
        return self.ref.L.ref_count_occupied(self.h, data.ctypes.data)

    def calibrate_unroll(self, words, cuckoo=False, min_s=0.25, seed=1):
        """The reference's unroll choice (blocked_bloomfilter_tune_impl.hpp:
        162-256; cuckoofilter_tune_impl.hpp:118-225): for u = 0, 1, 2, 4 (and 8
        for cuckoo filters), probe 32 Ki uniform random keys in 1024-key batches
        on one thread, repeatedly for at least 250 ms, against a zeroed filter
        of the same size (the reference does not insert before timing), and
        keep the u of the fewest time units per lookup.  `words` is the
        filter's word array; a zeroed copy of its size is timed.  Returns
        (u, {u: ns per lookup})."""
        rng = np.random.default_rng(seed)
        keys = rng.integers(0, 1 << 32, size=4 * 1024 * 8, dtype=np.uint64).astype(np.uint32)
        zero = np.zeros_like(words)
        zero[:] = 0   # touch the pages, as the reference's std::vector(size, 0) does
        out = np.zeros(len(keys) + 64, dtype=np.uint32)
        per = {}
        for u in ((0, 1, 2, 4, 8) if cuckoo else (0, 1, 2, 4)):
            reps = 0
            t0 = time.perf_counter()
            while True:
                self.ref.L.ref_batch_contains_mt(self.h, zero.ctypes.data, keys, len(keys), out, 1, u)
                reps += 1
                dt = time.perf_counter() - t0
                if dt > min_s:
                    break
            per[u] = dt * 1e9 / (reps * len(keys))
        return min(per, key=per.get), per


def try_reflib():
    try:
        return RefLib()
    except (FileNotFoundError, OSError):
        return None


class RefBcf:
    """The reference's dtl::bcf (oracle/_ref/libdtlref_bcf.so: plain x86-64,
    the scalar batch path; variant "avx2": the AVX2 batch path)."""

    def __init__(self, variant="scalar"):
        name = "libdtlref_bcf.so" if variant == "scalar" else f"libdtlref_bcf_{variant}.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.variant, self.path = variant, path
        L = C.CDLL(path)
        vp = C.c_void_p
        L.ref_bcf_create.restype = vp
        L.ref_bcf_create.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        L.ref_bcf_destroy.argtypes = [vp]
        L.ref_bcf_size.restype = C.c_uint64
        L.ref_bcf_size.argtypes = [vp]
        L.ref_bcf_size_in_bytes.restype = C.c_uint64
        L.ref_bcf_size_in_bytes.argtypes = [vp]
        L.ref_bcf_name.restype = C.c_size_t
        L.ref_bcf_name.argtypes = [vp, C.c_char_p, C.c_size_t]
        L.ref_bcf_batch_insert.restype = C.c_int
        L.ref_bcf_batch_insert.argtypes = [vp, vp, _u32p, C.c_uint32]
        L.ref_bcf_contains.restype = C.c_int
        L.ref_bcf_contains.argtypes = [vp, vp, C.c_uint32]
        L.ref_bcf_batch_contains.restype = C.c_uint64
        L.ref_bcf_batch_contains.argtypes = [vp, vp, _u32p, C.c_uint32, _u32p, C.c_uint32]
        L.ref_bcf_batch_contains_mt.restype = C.c_uint64
        L.ref_bcf_batch_contains_mt.argtypes = [vp, vp, _u32p, C.c_uint64, _u32p, C.c_int]
        L.ref_bcf_batch_contains_mt_list.restype = C.c_uint64
        L.ref_bcf_batch_contains_mt_list.argtypes = [vp, vp, _u32p, C.c_uint64, _u32p, C.c_int]
        self.L = L

    def create(self, m, block_bytes=64, t=16, a=4):
        h = self.L.ref_bcf_create(m, block_bytes, t, a)
        return _RefBcfFilter(self, h) if h else None


class _RefBcfFilter:
    def __init__(self, ref, h):
        self.ref, self.h = ref, h

    def __del__(self):
        try:
            self.ref.L.ref_bcf_destroy(self.h)
        except Exception:
            pass

    @property
    def size_u32(self):
        return self.ref.L.ref_bcf_size(self.h)

    @property
    def size_in_bytes(self):
        return self.ref.L.ref_bcf_size_in_bytes(self.h)

    def name(self):
        buf = C.create_string_buffer(512)
        self.ref.L.ref_bcf_name(self.h, buf, 512)
        return buf.value.decode()

    def alloc(self):
        # the reference's words, plus 64 bytes of slack for the AVX2 path's
        # 256-bit stores past the last match
        return np.zeros(self.size_u32 + 16, dtype=np.uint32)

    def insert(self, data, keys):
        k = _keys(keys)
        return bool(self.ref.L.ref_bcf_batch_insert(self.h, data.ctypes.data, k, len(k)))

    def contains(self, data, key):
        return bool(self.ref.L.ref_bcf_contains(self.h, data.ctypes.data, int(key)))

    def batch_contains(self, data, keys, match_offset=0):
        k = _keys(keys)
        out = np.zeros(len(k) + 16, dtype=np.uint32)
        n = self.ref.L.ref_bcf_batch_contains(self.h, data.ctypes.data, k, len(k), out, match_offset & 0xFFFFFFFF)
        return out[:n].copy()

    def batch_contains_mt(self, data, keys, threads, out=None):
        k = _keys(keys)
        if out is None:
            out = np.zeros(len(k) + 16, dtype=np.uint32)
        return self.ref.L.ref_bcf_batch_contains_mt(self.h, data.ctypes.data, k, len(k), out, threads)

    def batch_contains_mt_list(self, data, keys, threads, out=None):
        """batch_contains_mt, then the threads' slices joined: the ascending
        positions (match_offset 0) of every matching key, a view of `out`."""
        k = _keys(keys)
        if out is None:
            out = np.zeros(len(k) + 16, dtype=np.uint32)
        n = self.ref.L.ref_bcf_batch_contains_mt_list(self.h, data.ctypes.data, k, len(k), out, threads)
        return out[:n]


def try_refbcf(variant="scalar"):
    try:
        return RefBcf(variant)
    except (FileNotFoundError, OSError):
        return None


class RefCbf:
    """The reference's classic Bloom filter (oracle/_ref/libdtlref_cbf.so);
    its batch_contains has no SIMD path."""

    variant = "scalar"

    def __init__(self):
        path = os.path.join(HERE, "_ref", "libdtlref_cbf.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        L = C.CDLL(path)
        vp = C.c_void_p
        L.ref_cbf_create.restype = vp
        L.ref_cbf_create.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32]
        L.ref_cbf_destroy.argtypes = [vp]
        L.ref_cbf_size.restype = C.c_uint64
        L.ref_cbf_size.argtypes = [vp]
        L.ref_cbf_length.restype = C.c_uint64
        L.ref_cbf_length.argtypes = [vp]
        L.ref_cbf_batch_insert.restype = C.c_int
        L.ref_cbf_batch_insert.argtypes = [vp, vp, _u32p, C.c_uint32]
        L.ref_cbf_batch_contains.restype = C.c_uint64
        L.ref_cbf_batch_contains.argtypes = [vp, vp, _u32p, C.c_uint32, _u32p, C.c_uint32]
        L.ref_cbf_batch_contains_mt.restype = C.c_uint64
        L.ref_cbf_batch_contains_mt.argtypes = [vp, vp, _u32p, C.c_uint64, _u32p, C.c_int]
        L.ref_cbf_batch_contains_mt_list.restype = C.c_uint64
        L.ref_cbf_batch_contains_mt_list.argtypes = [vp, vp, _u32p, C.c_uint64, _u32p, C.c_int]
        self.L = L

    def create(self, k, m, magic=False):
        h = self.L.ref_cbf_create(m, k, 1 if magic else 0)
        return _RefCbfFilter(self, h) if h else None


class _RefCbfFilter:
    def __init__(self, ref, h):
        self.ref, self.h = ref, h

    def __del__(self):
        try:
            self.ref.L.ref_cbf_destroy(self.h)
        except Exception:
            pass

    @property
    def size_u32(self):
        return self.ref.L.ref_cbf_size(self.h)

    @property
    def length(self):
        return self.ref.L.ref_cbf_length(self.h)

    def alloc(self):
        return np.zeros(self.size_u32 + 16, dtype=np.uint32)

    def insert(self, data, keys):
        k = _keys(keys)
        return bool(self.ref.L.ref_cbf_batch_insert(self.h, data.ctypes.data, k, len(k)))

    def batch_contains(self, data, keys, match_offset=0):
        k = _keys(keys)
        out = np.zeros(len(k) + 16, dtype=np.uint32)
        n = self.ref.L.ref_cbf_batch_contains(self.h, data.ctypes.data, k, len(k), out, match_offset & 0xFFFFFFFF)
        return out[:n].copy()

    def batch_contains_mt(self, data, keys, threads, out=None):
        k = _keys(keys)
        if out is None:
            out = np.zeros(len(k) + 16, dtype=np.uint32)
        return self.ref.L.ref_cbf_batch_contains_mt(self.h, data.ctypes.data, k, len(k), out, threads)

    def batch_contains_mt_list(self, data, keys, threads, out=None):
        """batch_contains_mt, then the threads' slices joined: the ascending
        positions (match_offset 0) of every matching key, a view of `out`."""
        k = _keys(keys)
        if out is None:
            out = np.zeros(len(k) + 16, dtype=np.uint32)
        n = self.ref.L.ref_cbf_batch_contains_mt_list(self.h, data.ctypes.data, k, len(k), out, threads)
        return out[:n]


def try_refcbf():
    try:
        return RefCbf()
    except (FileNotFoundError, OSError):
        return None
