"""Analytic false-positive rates of the filter family, in numpy float64.

Restates the reference's formulas term for term:
  dtl::bloomfilter::fpr(m, n, config)     blocked_bloomfilter/fpr.hpp:12-61
    standard Bloom (m, n, k)              blocked_bloomfilter/math.hpp:17-24
    fpr_blocked (S == B, z == 1)          math.hpp:30-55
    fpr_blocked_sectorized (S < B, z == 1) math.hpp:61-88
    fpr_zoned + p_cache + p_load (z > 1)  math.hpp:91-145
  dtl::cuckoofilter::fpr                  math.hpp:198-205

B = block bits, S = sector bits = B / sector_cnt.  Self collisions are on
(the default of fpr(m, n, config)); the outer Poisson sum stops by the
reference's rule: term i is taken while (sum of the earlier weights) + 1e-5
< 1.  Boost's Poisson pmf is evaluated as exp(i ln(lam) - lam - lgamma(i+1)).

Every Bloom formula depends on m and n only through c = m / n (bits per key),
so a configuration's FPR is tabulated once as a function of c.
"""
import math

import numpy as np

EPSILON = 1e-5  # the epsilon fpr(m, n, ...) passes down (fpr.hpp:20)


def _lgamma_table(n):
    return np.array([math.lgamma(i + 1.0) for i in range(n)], dtype=np.float64)


_LG = _lgamma_table(4096)  # ln(i!) for i < 4096


def _poisson(lam, i):
    """pmf(i; lam) for lam (..., 1) and integer i (I,), lam > 0."""
    lam = np.asarray(lam, dtype=np.float64)
    return np.exp(i * np.log(lam) - lam - _LG[i])


def std_fpr(m, n, k):
    """Standard Bloom filter: (1 - (1 - 1/m)^(k n))^k   (math.hpp:17-24)."""
    return np.power(1.0 - np.power(1.0 - 1.0 / m, k * np.asarray(n, dtype=np.float64)), k)


def _outer_sum(lam, inner):
    """sum_i pmf(i; lam) * inner[i] with the reference's stopping rule, for an
    array of lam; inner must cover every i the rule can reach."""
    lam = np.atleast_1d(np.asarray(lam, dtype=np.float64))[:, None]
    i = np.arange(len(inner))
    d = _poisson(lam, i)
    before = np.cumsum(d, axis=1) - d           # weight summed before term i (sequential)
    take = (before + EPSILON) < 1.0
    if take[:, -1].any():
        raise ValueError("Poisson sum needs more terms than tabulated")
    return np.sum(np.where(take, d * inner, 0.0), axis=1)


def _terms_for(lam_max):
    return int(lam_max + 12.0 * math.sqrt(lam_max) + 40)


class BloomFpr:
    """FPR of one blocked Bloom configuration as a function of bits per key."""

    def __init__(self, k, word_size, word_cnt, sector_cnt=1, zone_cnt=1, self_collisions=True):
        self.k = float(k)
        self.B = word_size * 8 * word_cnt
        self.S = self.B // sector_cnt
        self.z = zone_cnt
        self.self_collisions = self_collisions
        self._inner = None

    def _inner_terms(self, n_terms):
        if self._inner is not None and len(self._inner) >= n_terms:
            return self._inner[:n_terms]
        B, S, z, k = float(self.B), float(self.S), self.z, self.k
        i = np.arange(n_terms, dtype=np.float64)
        if self.S == self.B and z == 1:                    # fpr_blocked
            k_act = B * (1.0 - (1.0 - 1.0 / B) ** k) if self.self_collisions else k
            inner = std_fpr(B, i, k_act)
        elif self.S < self.B and z == 1:                   # fpr_blocked_sectorized
            s = B / S
            kps = k / s
            if self.self_collisions:
                kps = S * (1.0 - (1.0 - 1.0 / S) ** kps)
            inner = np.power(std_fpr(S, i, kps), s)
        elif self.S < self.B and z > 1:                    # fpr_zoned: p_cache(z, S, B, k, i)
            kpz = k / z                                    # p_cache divides k by z, uncorrected
            inner = np.zeros(n_terms)
            j = np.arange(1, n_terms, dtype=np.float64)
            f_mini = std_fpr(S, j, kpz)                    # fpr(S, j, k/z), j >= 1
            ji = np.arange(1, n_terms)
            for ii in range(1, n_terms):
                ev = ii * z * S / B
                p_l = np.exp(ji[:ii] * math.log(ev) - ev - _LG[ji[:ii]])
                inner[ii] = np.sum(p_l * f_mini[:ii]) ** z
        else:
            raise ValueError(f"invalid blocked Bloom filter configuration: B={self.B}, S={self.S}, z={z}")
        self._inner = inner
        return inner

    def __call__(self, bits_per_key):
        """FPR at c = m / n bits per key (array or scalar)."""
        c = np.atleast_1d(np.asarray(bits_per_key, dtype=np.float64))
        lam = self.B / c
        inner = self._inner_terms(_terms_for(float(lam.max())))
        out = _outer_sum(lam, inner)
        return out if np.ndim(bits_per_key) else float(out[0])


def bloom_fpr(m, n, k, word_size, word_cnt, sector_cnt=1, zone_cnt=1):
    """dtl::bloomfilter::fpr(m, n, config) for one (m, n)."""
    return BloomFpr(k, word_size, word_cnt, sector_cnt, zone_cnt)(m / n)


def cuckoo_fpr(tags_per_bucket, bits_per_tag, load_factor):
    """1 - (1 - 1/(2^t - 1))^(2 b lf)   (math.hpp:198-205, the counting variant)."""
    return 1.0 - np.power(1.0 - 1.0 / (2.0 ** bits_per_tag - 1.0),
                          2.0 * tags_per_bucket * np.asarray(load_factor, dtype=np.float64))
