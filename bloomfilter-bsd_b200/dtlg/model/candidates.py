"""The configuration candidates the cost model chooses among.

Bloom candidates follow the reference's enumeration of valid configurations
(model/util.hpp:17-64): k 1..16, word size 4 or 8 bytes, 1..16 words per block
with blocks of at most 64 bytes, sector_cnt dividing k and at most the word
count, and zoned layouts (sector_cnt = word_cnt >= 4, zone_cnt < word_cnt,
zone_cnt dividing k).  Sectors are limited to 1..8 and zones to 2..4.  The
addressing mode is not a candidate dimension: a filter of m bits uses MAGIC
addressing unless its block count is a power of two (blocked_bloomfilter.hpp:
234-242), and calibration times the MAGIC form.

Cuckoo candidates (model/util.hpp:70-84): 8, 12 or 16 bits per tag, 2 or 4
tags per bucket.  A cuckoo table can be filled up to the load factor that
partial-key cuckoo hashing with two buckets reaches (about 84 % with 2 slots
per bucket, 95 % with 4); its size in bits per key is therefore at least
t / lf_max, and its FPR follows the load factor actually used.
"""
from dataclasses import dataclass

import numpy as np

from .fpr import BloomFpr, cuckoo_fpr

CUCKOO_MAX_LOAD = {2: 0.84, 4: 0.95}


@dataclass(frozen=True)
class Candidate:
    kind: str              # "bloom" or "cuckoo"
    word_size: int = 0     # bloom: bytes per word
    w: int = 0             # bloom: words per block
    s: int = 0             # bloom: sectors
    z: int = 0             # bloom: zones
    k: int = 0             # bloom: hash functions
    t: int = 0             # cuckoo: bits per tag
    b: int = 0             # cuckoo: tags per bucket

    @property
    def name(self):
        if self.kind == "cuckoo":
            return f"cf t={self.t} b={self.b}"
        return f"bbf u{self.word_size * 8} w={self.w} s={self.s} z={self.z} k={self.k}"

    @property
    def block_bytes(self):
        return self.word_size * self.w if self.kind == "bloom" else (self.t * self.b + 7) // 8

    def min_bits_per_key(self):
        return self.t / CUCKOO_MAX_LOAD[self.b] if self.kind == "cuckoo" else 0.0

    def fpr(self, bits_per_key):
        """FPR at the given bits per key (inf where the layout cannot hold the keys)."""
        c = np.asarray(bits_per_key, dtype=np.float64)
        if self.kind == "bloom":
            return BloomFpr(self.k, self.word_size, self.w, self.s, self.z)(c)
        lf = self.t / c
        return np.where(lf <= CUCKOO_MAX_LOAD[self.b] + 1e-12, cuckoo_fpr(self.b, self.t, np.minimum(lf, 1.0)),
                        np.inf)

    def config(self):
        """The dtlg config object (construct(config, m) builds the filter)."""
        from .. import blocked_bloomfilter_config, cuckoofilter_config
        if self.kind == "cuckoo":
            return cuckoofilter_config(bits_per_tag=self.t, tags_per_bucket=self.b)
        return blocked_bloomfilter_config(k=self.k, word_size=self.word_size, word_cnt_per_block=self.w,
                                          sector_cnt=self.s, zone_cnt=self.z)


def bloom_candidates(max_sectors=8, zones=(2, 4)):
    out = []
    for word_size in (4, 8):
        for w in (1, 2, 4, 8, 16):
            if word_size * w > 64:
                continue
            for k in range(1, 17):
                for s in (1, 2, 4, 8, 16):
                    if s > w or s > k or k % s or s > max_sectors:
                        continue
                    out.append(Candidate("bloom", word_size, w, s, 1, k))
                if w >= 4:
                    for z in zones:
                        if z >= w or z > k or k % z:
                            continue
                        out.append(Candidate("bloom", word_size, w, w, z, k))
    return out


def cuckoo_candidates(tags=(8, 12, 16), buckets=(2, 4)):
    return [Candidate("cuckoo", t=t, b=b) for t in tags for b in buckets]


def all_candidates():
    return bloom_candidates() + cuckoo_candidates()


def by_name(name):
    for c in all_candidates():
        if c.name == name:
            return c
    raise KeyError(name)
