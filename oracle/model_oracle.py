"""Oracle of the configuration-choice path (TEST INFRASTRUCTURE ONLY).

Used by tests/ as the oracle; the product never imports it.

  * FPR formulas as plain Python loops, step for step as the reference writes
    them (src/dtl/filter/blocked_bloomfilter/fpr.hpp:12-61, math.hpp:17-205),
    with Boost's Poisson pmf restated as exp(i ln(lam) - lam - lgamma(i+1)).
    The reference's own code is the stronger pin where it compiles here
    (oracle/_ref/libdtlref_fpr.so); these loops stand in elsewhere.
  * The calibrated cost search as a plain loop over candidates and bits per
    key (the product's search is native, csrc/cost_search.cpp).
  * The MLP in float64 numpy: forward pass, weighted squared-error loss,
    backward pass and one Adam step, in the product's parameter layout
    (per layer W [in x out] row-major, then b [out]).
"""
import math

import numpy as np

# ---------------------------------------------------------------- FPR (math.hpp)


def poisson_pmf(lam, i):
    return math.exp(i * math.log(lam) - lam - math.lgamma(i + 1.0))


def std_fpr(m, n, k):
    """math.hpp:17-24."""
    return math.pow(1.0 - math.pow(1.0 - 1.0 / m, k * n), k)


def fpr_blocked(m, n, k, B, self_collisions, epsilon):
    """math.hpp:30-55."""
    f = 0.0
    c = m / n
    lam = B / c
    k_act = B * (1.0 - math.pow(1.0 - 1.0 / B, k)) if self_collisions else k
    d_sum, i = 0.0, 0
    while d_sum + epsilon < 1.0:
        d = poisson_pmf(lam, i)
        d_sum += d
        f += d * std_fpr(B, i, k_act)
        i += 1
    return f


def fpr_blocked_sectorized(m, n, k, B, S, self_collisions, epsilon):
    """math.hpp:61-88."""
    f = 0.0
    c = m / n
    lam = B / c
    s = B / S
    k_per_s = k / s
    if self_collisions:
        k_per_s = S * (1.0 - math.pow(1.0 - 1.0 / S, k_per_s))
    d_sum, i = 0.0, 0
    while d_sum + epsilon < 1.0:
        d = poisson_pmf(lam, i)
        d_sum += d
        f += d * math.pow(std_fpr(S, i, k_per_s), s)
        i += 1
    return f


def p_cache(s, S, B, k, i):
    """math.hpp:99-115."""
    k_per_s = k / s
    total = 0.0
    for j in range(1, i + 1):
        ev = i * s * S / B
        total += poisson_pmf(ev, j) * std_fpr(S, j, k_per_s)
    return math.pow(total, s)


def fpr_zoned(m, n, k, B, S, z, epsilon):
    """math.hpp:117-145 (its self-collision correction is computed but unused)."""
    f = 0.0
    c = m / n
    lam = B / c
    d_sum, i = 0.0, 0
    while d_sum + epsilon < 1.0:
        d = poisson_pmf(lam, i)
        d_sum += d
        f += d * p_cache(z, S, B, k, i)
        i += 1
    return f


def bbf_fpr(m, n, k, word_size, w, s, z):
    """fpr(m, n, config) (fpr.hpp:12-61): epsilon 1e-5, self collisions on."""
    B = word_size * 8 * w
    S = B // s
    if S == B and z == 1:
        return fpr_blocked(m, n, k, B, True, 1e-5)
    if S < B and z == 1:
        return fpr_blocked_sectorized(m, n, k, B, S, True, 1e-5)
    if S < B and z > 1:
        return fpr_zoned(m, n, k, B, S, z, 1e-5)
    raise ValueError("invalid configuration")


def cf_fpr(tags_per_bucket, bits_per_tag, load_factor):
    """math.hpp:198-205."""
    return 1.0 - math.pow(1.0 - 1.0 / (math.pow(2.0, bits_per_tag) - 1.0), 2.0 * tags_per_bucket * load_factor)


# ---------------------------------------------------------------- cost search


def lookup_ns(ns_row, first, step, log2_bytes):
    S = len(ns_row)
    if S == 1:
        return ns_row[0]
    x = min(max((log2_bytes - first) / step, 0.0), S - 1.0)
    i = min(int(x), S - 2)
    f = x - i
    return ns_row[i] * (1.0 - f) + ns_row[i + 1] * f


def search(bpk, fpr, first, step, ns, ns_per_match, budget, q, ns_second=None):
    """One query q = (log2_n, fpr_target, hit_ratio, work_ns, l2_resident):
    (best index or -1, best cost, per-candidate best costs).  ns_second: the
    added time of a block's second half, paid by members and by the
    non-members that pass the first half (probability sqrt(f))."""
    log2_n, target, h, work, l2 = q
    n = 2.0 ** log2_n
    best, best_cost, per = -1, math.inf, []
    for c in range(len(fpr)):
        cc = math.inf
        for k in range(len(bpk)):
            f = fpr[c][k]
            if not f <= target:
                continue
            if l2 and n * bpk[k] / 8.0 > budget:
                continue
            lb = log2_n + math.log2(bpk[k]) - 3.0
            t = lookup_ns(ns[c], first, step, lb)
            if ns_second is not None:
                t += (h + (1 - h) * min(1.0, math.sqrt(max(0.0, f)))) * lookup_ns(ns_second[c], first, step, lb)
            cost = t + ns_per_match * (h + (1 - h) * f) + work * (1 - h) * f
            cc = min(cc, cost)
        per.append(cc)
        if cc < best_cost:
            best, best_cost = c, cc
    return best, best_cost, per


# ---------------------------------------------------------------- MLP (float64)


def layers(flat, dims):
    out, off = [], 0
    for a, b in zip(dims[:-1], dims[1:]):
        W = np.asarray(flat[off:off + a * b], dtype=np.float64).reshape(a, b)
        off += a * b
        out.append((W, np.asarray(flat[off:off + b], dtype=np.float64)))
        off += b
    return out


def forward(flat, dims, x):
    acts = []
    h = np.asarray(x, dtype=np.float64)
    L = len(dims) - 1
    for i, (W, b) in enumerate(layers(flat, dims)):
        h = h @ W + b
        if i < L - 1:
            h = np.maximum(h, 0.0)
        acts.append(h)
    return acts


def loss_grad(flat, dims, x, t, w):
    """L = (1/N) sum w (y - t)^2 and its gradient in the flat layout."""
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    N = x.shape[0]
    acts = forward(flat, dims, x)
    d = acts[-1] - t
    loss = float(np.sum(w * d * d) / N)
    dz = 2.0 / N * w * d
    grads = []
    lay = layers(flat, dims)
    for i in range(len(lay) - 1, -1, -1):
        inp = x if i == 0 else acts[i - 1]
        grads.append((inp.T @ dz, dz.sum(axis=0)))
        if i > 0:
            dz = (dz @ lay[i][0].T) * (acts[i - 1] > 0)
    grads.reverse()
    return loss, np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])


def adam(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba, 2015); t counts from 1."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p, m, v
