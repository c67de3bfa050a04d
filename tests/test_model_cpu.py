"""The configuration-choice path on the CPU: analytic FPR against the
reference's own formulas (compiled from its sources, where present) and the
oracle's loops, against the false-positive rate the filters really have, and
the native exhaustive search against the oracle's plain loop."""
import ctypes as C
import math
import os

import numpy as np
import pytest

import model_oracle as MO
import oracle as O
from dtlg import keygen
from dtlg.model import cost as CM
from dtlg.model.calibration import DEFAULT_LOG2_BYTES, DEFAULT_PATH, CalibrationData
from dtlg.model.candidates import all_candidates, bloom_candidates
from dtlg.model.fpr import BloomFpr, cuckoo_fpr

REF_FPR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libdtlref_fpr.so")


def ref_fpr_lib():
    if not os.path.exists(REF_FPR):
        return None
    L = C.CDLL(REF_FPR)
    L.ref_bbf_fpr.restype = C.c_double
    L.ref_bbf_fpr.argtypes = [C.c_uint64, C.c_uint64] + [C.c_uint32] * 5
    L.ref_cf_fpr.restype = C.c_double
    L.ref_cf_fpr.argtypes = [C.c_uint32, C.c_uint32, C.c_double]
    return L


@pytest.mark.skipif(ref_fpr_lib() is None, reason="oracle/_ref/libdtlref_fpr.so not built")
def test_fpr_matches_reference_formulas_every_candidate():
    L = ref_fpr_lib()
    n = 1 << 20
    bpk = np.array([1.0, 2.5, 4.0, 7.3, 12.0, 16.0, 23.9, 40.0])
    worst = 0.0
    for c in bloom_candidates():
        ref = np.array([L.ref_bbf_fpr(int(round(n * b)), n, c.k, c.word_size, c.w, c.s, c.z) for b in bpk])
        # the reference sees the integer m; restate at the same m / n
        mine = c.fpr(np.array([int(round(n * b)) / n for b in bpk]))
        rel = np.abs(mine - ref) / np.maximum(ref, 1e-300)
        worst = max(worst, float(rel.max()))
    assert worst < 1e-9, worst
    for b in (2, 4):
        for t in (8, 12, 16):
            for lf in (0.5, 0.84, 0.95):
                assert math.isclose(float(cuckoo_fpr(b, t, lf)), L.ref_cf_fpr(b, t, lf), rel_tol=1e-12)


def test_fpr_matches_oracle_loops():
    for c in bloom_candidates()[::9]:
        for bpk in (3.0, 10.0, 20.0):
            m, n = int(bpk * 4096), 4096
            want = MO.bbf_fpr(m, n, c.k, c.word_size, c.w, c.s, c.z)
            got = BloomFpr(c.k, c.word_size, c.w, c.s, c.z)(m / n)
            assert math.isclose(got, want, rel_tol=1e-9, abs_tol=1e-300), (c.name, bpk)


def test_poisson_pmf_against_mpmath():
    mpmath = pytest.importorskip("mpmath")
    for lam in (0.3, 4.0, 37.5, 256.0):
        for i in (0, 1, 7, 40, 300):
            want = float(mpmath.e ** (-lam) * mpmath.mpf(lam) ** i / mpmath.factorial(i))
            got = MO.poisson_pmf(lam, i)
            assert math.isclose(got, want, rel_tol=1e-9, abs_tol=1e-300)


@pytest.mark.parametrize("cfg", [(8, 8, 8, 1, 8), (8, 8, 8, 2, 8), (8, 8, 8, 4, 8), (4, 16, 16, 2, 8),
                                 (4, 1, 1, 1, 4), (4, 4, 1, 1, 4)])
def test_analytic_fpr_tracks_measured_fpr(cfg):
    """The model's FPR against the rate a bit-exact filter really shows (the
    oracle build, 2^16 keys, 2^21 non-member probes)."""
    wb, w, s, z, k = cfg
    n = 1 << 16
    for bpk in (8, 16):
        ob = O.Bloom(wb, w, s, z, k, n * bpk + 1000)
        d = ob.alloc()
        ob.insert(d, keygen.build_keys(n, 5))
        pk, _ = keygen.probe_keys(n, 1 << 21, 0.0, 5)
        measured = len(ob.batch_contains(d, pk, 0)) / len(pk)
        analytic = BloomFpr(k, wb, w, s, z)(ob.m_actual / n)
        assert abs(measured / analytic - 1.0) < 0.12, (cfg, bpk, measured, analytic)


def test_candidate_set():
    cands = all_candidates()
    assert len(cands) == 284 and len({c.name for c in cands}) == 284
    for c in cands:
        if c.kind == "bloom" and c.z == 1:
            assert c.k % c.s == 0 and c.s <= c.w and c.block_bytes <= 64 and c.s <= 8
        elif c.kind == "bloom":
            assert c.s == c.w >= 4 and c.z < c.w and c.z <= 4 and c.k % c.z == 0 and c.block_bytes <= 64
    assert sum(c.kind == "cuckoo" for c in cands) == 6


def test_every_candidate_constructs():
    from dtlg import construct
    from dtlg.model.calibration import _magic_bits
    for c in all_candidates():
        f = construct(c.config(), _magic_bits(2 ** 20.3, c))
        assert f.alloc_words() > 0 and f.is_magic()


def small_model(seed=3, C_=7, K=20, S=9):
    rng = np.random.default_rng(seed)
    bpk = np.sort(rng.uniform(1, 30, K))
    fpr = np.sort(rng.uniform(1e-6, 0.2, (C_, K)), axis=1)[:, ::-1].copy()
    fpr[1, :4] = np.inf
    ns = rng.uniform(0.005, 0.05, (C_, S))
    cal = CalibrationData([all_candidates()[i] for i in range(C_)], 12.0 + 2.0 * np.arange(S), ns, 0.003, {})
    m = CM.CostModel(cal, l2_budget_bytes=1 << 20, bpk_grid=bpk)
    m.fpr = np.ascontiguousarray(fpr)                 # synthetic FPR tables
    m.tables.fpr = C.c_void_p(m.fpr.ctypes.data)
    return m, bpk, fpr, ns


def test_native_search_matches_oracle_loop():
    m, bpk, fpr, ns = small_model()
    q = CM.sample_queries(300, 5)
    q["log2_n"] = np.random.default_rng(1).uniform(8, 22, len(q))
    r = m.search(q, per_candidate=True, threads=3)
    for i in range(len(q)):
        b, bc, per = MO.search(bpk, fpr, 12.0, 2.0, ns, 0.003, 1 << 20, tuple(q[i])[:5])
        assert r["best"][i] == b
        if b >= 0:
            assert math.isclose(r["best_cost"][i], bc, rel_tol=1e-12)
        np.testing.assert_allclose(r["cand_cost"][i], per, rtol=1e-12)
    # evaluating the search's own choice reproduces its cost
    ok = r["best"] >= 0
    k = np.array([np.nonzero(bpk == b)[0][0] for b in r["best_bpk"][ok]])
    np.testing.assert_allclose(m.evaluate(q[ok], r["best"][ok], k), r["best_cost"][ok], rtol=1e-12)


def test_native_search_with_second_half_matches_oracle_loop():
    """The second half of a block: the native search and the oracle's loop
    agree when the calibration carries it."""
    m, bpk, fpr, ns = small_model()
    ns2 = np.random.default_rng(9).uniform(0.0, 0.03, ns.shape)
    m.ns_second = np.ascontiguousarray(ns2)
    m.tables.ns_second = C.c_void_p(m.ns_second.ctypes.data)
    q = CM.sample_queries(300, 6)
    q["log2_n"] = np.random.default_rng(2).uniform(8, 22, len(q))
    r = m.search(q, per_candidate=True, threads=2)
    for i in range(len(q)):
        b, bc, per = MO.search(bpk, fpr, 12.0, 2.0, ns, 0.003, 1 << 20, tuple(q[i])[:5], ns_second=ns2)
        assert r["best"][i] == b
        np.testing.assert_allclose(r["cand_cost"][i], per, rtol=1e-12)


def test_loaded_filter_costs_more_at_few_bits_per_key():
    """A filter with few bits per key has most of its bits set, so many
    non-members pass the first half of a block and load the second: priced
    on a zeroed filter (the first half only) such a candidate looks cheaper
    than it is.  With the second half in the tables the low-bits/key cost
    rises by (h + (1 - h) sqrt(f)) * second half, the high-bits/key one barely."""
    m, bpk, fpr, ns = small_model()
    q = CM.make_queries([16.0] * 2, [1.0] * 2, [0.0] * 2, [5.0] * 2, [0] * 2)
    c = np.array([0, 0], dtype=np.int32)
    k = np.array([0, len(bpk) - 1], dtype=np.uint32)   # fewest and most bits per key
    zeroed = m.evaluate(q, c, k)
    ns2 = np.full(ns.shape, 0.02)
    m.ns_second = np.ascontiguousarray(ns2)
    m.tables.ns_second = C.c_void_p(m.ns_second.ctypes.data)
    loaded = m.evaluate(q, c, k)
    want = np.sqrt(fpr[0, k]) * 0.02
    np.testing.assert_allclose(loaded - zeroed, want, rtol=1e-12)
    assert (loaded - zeroed)[0] > 5 * (loaded - zeroed)[1]


def test_repair_moves_to_the_nearest_feasible_size():
    m, bpk, fpr, ns = small_model()
    q = CM.make_queries([16.0, 16.0], [fpr[2, 10], 1.0], [0.1, 0.1], [50.0, 50.0], [0, 1])
    k, ok = m.repair(q, np.array([2, 2]), np.array([0, len(bpk) - 1]))
    assert ok.all() and k[0] == 10
    assert 2 ** 16 * bpk[k[1]] / 8 <= 1 << 20 and (k[1] == len(bpk) - 1 or 2 ** 16 * bpk[k[1] + 1] / 8 > 1 << 20)


@pytest.mark.skipif(not os.path.exists(DEFAULT_PATH), reason="no calibration data")
def test_committed_calibration_data():
    cal = CalibrationData.load()
    assert [c.name for c in cal.candidates] == [c.name for c in all_candidates()]
    assert np.allclose(cal.log2_bytes, DEFAULT_LOG2_BYTES)
    assert cal.ns_per_key.shape == (284, len(DEFAULT_LOG2_BYTES))
    assert np.isfinite(cal.ns_per_key).all() and (cal.ns_per_key > 0).all()
    assert cal.meta["runs"] >= 20000
    # probes of DRAM-resident filters cost more than of L2-resident ones
    big, small = cal.ns_per_key[:, -1], cal.ns_per_key[:, 20]
    assert np.median(big / small) > 1.5


@pytest.mark.skipif(not os.path.exists(DEFAULT_PATH), reason="no calibration data")
def test_committed_calibration_prices_the_second_half():
    """The committed GPU calibration times every layout on a zeroed and on a
    half-filled filter.  Blocks that are tested in two halves (64-byte
    sectorized) pay a second half that a zeroed filter never shows; one-word
    blocks have none.  A sectorized filter at few bits per key (most bits
    set, so many non-members pass the first half) is then priced well above
    its zeroed-filter cost, one at many bits per key barely above it."""
    cal = CalibrationData.load()
    assert cal.ns_second is not None and cal.ns_second.shape == cal.ns_per_key.shape
    assert (cal.ns_second >= 0).all() and np.isfinite(cal.ns_second).all()
    names = [c.name for c in cal.candidates]
    sect, one = names.index("bbf u64 w=8 s=8 z=1 k=8"), names.index("bbf u32 w=1 s=1 z=1 k=4")
    l2 = (cal.log2_bytes >= 16) & (cal.log2_bytes <= 26)       # 64 KiB .. 64 MiB
    assert cal.ns_second[sect, l2].mean() > 0.2 * cal.ns_per_key[sect, l2].mean()
    assert cal.ns_second[one].max() < 0.1 * cal.ns_per_key[one].min()     # timing noise only
    loaded = CM.CostModel(cal)
    zeroed = CM.CostModel(CalibrationData(cal.candidates, cal.log2_bytes, cal.ns_per_key, cal.ns_per_match,
                                          cal.meta))
    # no downstream work: the cost is the probe time plus the match writes
    q = CM.make_queries([20.0, 20.0], [1.0, 1.0], [0.0, 0.0], [0.0, 0.0], [0, 0])
    k = loaded.bpk_index([4.0, 24.0]).astype(np.uint32)
    c = np.array([sect, sect], dtype=np.int32)
    lo, hi = loaded.evaluate(q, c, k), zeroed.evaluate(q, c, k)
    probe0 = hi - cal.ns_per_match * loaded.fpr[sect, k]   # zeroed-filter probe time
    assert lo[0] - hi[0] > 0.15 * probe0[0]       # 4 bits per key: the second half is paid often
    assert lo[1] - hi[1] < 0.05 * probe0[1]       # 24 bits per key: rarely


@pytest.mark.skipif(not os.path.exists(DEFAULT_PATH), reason="no calibration data")
def test_skyline_and_search_on_committed_data():
    model = CM.CostModel(CalibrationData.load())
    q = CM.feasible_queries(model, 300, 4)
    r = model.search(q)
    assert (r["best"] >= 0).all() and np.isfinite(r["best_cost"]).all()
    sky = CM.Skyline(model)
    cand, bpk = sky.lookup(q)
    k, ok = model.repair(q, cand, model.bpk_index(bpk))
    cost = model.evaluate(q[ok], cand[ok], k[ok])
    assert (cost >= r["best_cost"][ok] * (1 - 1e-12)).all()   # nothing beats the exhaustive search


def test_mlp_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    dims = [5, 8, 8, 6]
    n_params = sum(a * b + b for a, b in zip(dims[:-1], dims[1:]))
    p = rng.normal(0, 0.5, n_params)
    x, t, w = rng.normal(size=(13, 5)), rng.normal(size=(13, 6)), rng.uniform(0, 1, (13, 6))
    _, g = MO.loss_grad(p, dims, x, t, w)
    eps = 1e-6
    for i in rng.choice(n_params, 40, replace=False):
        e = np.zeros(n_params)
        e[i] = eps
        num = (MO.loss_grad(p + e, dims, x, t, w)[0] - MO.loss_grad(p - e, dims, x, t, w)[0]) / (2 * eps)
        assert math.isclose(num, g[i], rel_tol=1e-5, abs_tol=1e-8)
