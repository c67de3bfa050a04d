"""Seeded synthetic key sets for builds and probes.

The reference publishes no dataset; its own benchmark probes uniform random
u32 keys (model/benchmark.cpp:20,82-95).  Here every key is the image of a
counter under a keyed bijection of [0, 2^32), so that

* the build set ``perm(0 .. n-1)`` has no duplicates, and
* a non-member ``perm(n + i)`` is guaranteed absent from the build set
  (with plain uniform draws a 2^28-key build would collide with 1/16 of the
  "misses").

Hits are drawn uniformly, with replacement, from the build set.  All of it is
pure uint64 numpy arithmetic, so the same seed gives the same keys on every
machine and numpy version.
"""
import numpy as np

_M64 = np.uint64(0xFFFFFFFF)


def _mix32(x, seed):
    """A bijection of u32 values (keyed odd multiplies and xorshifts)."""
    s = np.uint64(seed & 0xFFFFFFFF)
    x = x.astype(np.uint64, copy=False)
    x = (x + s * np.uint64(0x9E3779B9)) & _M64
    x = (x * np.uint64(0x85EBCA6B)) & _M64
    x ^= x >> np.uint64(13)
    x = (x * np.uint64(0xC2B2AE35)) & _M64
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(((0x27D4EB2F ^ (seed * 2)) | 1) & 0xFFFFFFFF)) & _M64
    x ^= x >> np.uint64(15)
    return x


def perm(idx, seed):
    """Image of the counters ``idx`` under the seeded bijection (uint32)."""
    return _mix32(np.asarray(idx, dtype=np.uint64), seed).astype(np.uint32)


def build_keys(n, seed, start=0):
    """The n distinct build keys perm(start .. start+n-1)."""
    return perm(np.arange(start, start + n, dtype=np.uint64), seed)


def probe_keys(n_build, n_probe, hit_ratio, seed, start=0, chunk=1 << 24):
    """n_probe probe keys; each is a build key with probability ``hit_ratio``
    (uniform over the build set) and otherwise a guaranteed non-member.

    Returns (keys, is_member) for probe indices start .. start+n_probe-1, so a
    probe stream can be produced in slices that concatenate exactly.
    """
    assert n_build + start + n_probe <= (1 << 32), "counter space exhausted"
    keys = np.empty(n_probe, dtype=np.uint32)
    member = np.empty(n_probe, dtype=bool)
    thr = np.uint64(int(hit_ratio * (1 << 32)))
    for b in range(0, n_probe, chunk):
        e = min(n_probe, b + chunk)
        i = np.arange(start + b, start + e, dtype=np.uint64)
        r = _mix32(i, seed ^ 0x5EED1)             # hit / miss coin
        hit = r < thr if n_build > 0 else np.zeros(e - b, dtype=bool)
        j = _mix32(i, seed ^ 0xB10C) % np.uint64(max(1, n_build))  # which member
        miss_ctr = np.uint64(n_build) + i
        src = np.where(hit, j, miss_ctr)
        keys[b:e] = _mix32(src, seed).astype(np.uint32)
        member[b:e] = hit
    return keys, member


def _mix32_torch(x, seed):
    """_mix32 on an int64 torch tensor (values < 2^32), bit-identical."""
    m = 0xFFFFFFFF
    s = seed & 0xFFFFFFFF
    x = (x + ((s * 0x9E3779B9) & m)) & m
    x = (x * 0x85EBCA6B) & m
    x ^= x >> 13
    x = (x * 0xC2B2AE35) & m
    x ^= x >> 16
    x = (x * ((((0x27D4EB2F ^ (seed * 2)) | 1)) & m)) & m
    x ^= x >> 15
    return x


def build_keys_torch(n, seed, device="cuda", start=0):
    """build_keys on the device (int32 tensor holding the uint32 keys)."""
    import torch
    i = torch.arange(start, start + n, dtype=torch.int64, device=device)
    return _to_i32(_mix32_torch(i, seed))


def probe_keys_torch(n_build, n_probe, hit_ratio, seed, start=0, device="cuda", chunk=1 << 26):
    """probe_keys on the device; returns (int32 keys, bool member)."""
    import torch
    assert n_build + start + n_probe <= (1 << 32), "counter space exhausted"
    keys = torch.empty(n_probe, dtype=torch.int32, device=device)
    member = torch.empty(n_probe, dtype=torch.bool, device=device)
    thr = int(hit_ratio * (1 << 32))
    for b in range(0, n_probe, chunk):
        e = min(n_probe, b + chunk)
        i = torch.arange(start + b, start + e, dtype=torch.int64, device=device)
        r = _mix32_torch(i.clone(), seed ^ 0x5EED1)
        hit = (r < thr) if n_build > 0 else torch.zeros_like(r, dtype=torch.bool)
        j = _mix32_torch(i.clone(), seed ^ 0xB10C) % max(1, n_build)
        src = torch.where(hit, j, i + n_build)
        keys[b:e] = _to_i32(_mix32_torch(src, seed))
        member[b:e] = hit
    return keys, member


def _to_i32(x):
    import torch
    return torch.where(x >= (1 << 31), x - (1 << 32), x).to(torch.int32)


def uniform_keys(n, seed):
    """n distinct keys spread uniformly over u32, standing in for the unique
    random keys of the reference's calibration runs (model/benchmark.cpp:82-95)."""
    return perm(np.arange(n, dtype=np.uint64), seed ^ 0xC0FFEE)
