"""The calibrated cost model and its exhaustive search (host side).

A query asks for the filter that minimises the cost per probed key

    cost(c, bpk) = t_c(n * bpk / 8 bytes, f, h) + ns_per_match * (h + (1 - h) * f)
                   + work_ns * (1 - h) * f,            f = fpr_c(bpk),

    t_c(size, f, h) = first_c(size) + (h + (1 - h) * sqrt(f)) * second_c(size),

subject to f <= fpr_target and, for an L2-resident query, a filter of at most
l2_budget_bytes.  first_c and second_c come from the GPU calibration runs:
the probe tests the first half of a block and loads the second half only for
keys that pass it -- every member, and a non-member with probability about
sqrt(f) -- so a filter with fewer bits per key (more bits set) pays the second
half more often.  This is the
reference's overhead = t_lookup(m) + tw * fpr(m, n, c) (model/cost_fn.hpp:
150-160) minimised over m for every configuration (model/optimizer.hpp:25-140,
tool/calibration/src/skyline_matrix_builder.cpp:88-115), with two query terms
the reference leaves implicit: the hit ratio (only non-members can be false
positives, and every match costs an output write) and the FPR target.

The search itself is native (dtlg_cost_search in libdtlg.so, all host cores);
bits per key run over a log-spaced grid from 1 to 50 (32 points per octave).

The skyline matrix is the reference's cached form of the search
(model/skyline_matrix.hpp:22-162): the best configuration precomputed on a grid
of query points and looked up by the next grid point in every dimension.
"""
import ctypes as C
import time

import numpy as np

from .. import _lib
from .calibration import CalibrationData

BPK_STEPS_PER_OCTAVE = 32
BPK_GRID = 2.0 ** (np.arange(0, 181) / BPK_STEPS_PER_OCTAVE)   # 1 .. 50.2 bits per key
L2_BUDGET_BYTES = 96 << 20

QUERY_DTYPE = np.dtype([("log2_n", "f8"), ("fpr_target", "f8"), ("hit_ratio", "f8"), ("work_ns", "f8"),
                        ("l2_resident", "u4"), ("_pad", "u4")])

# the query space the model is trained and evaluated on
LOG2_N_RANGE = (10.0, 28.0)
FPR_RANGE = (1e-5, 1e-1)
HIT_RANGE = (0.0, 0.9)
WORK_NS_RANGE = (5.0, 500.0)


def make_queries(log2_n, fpr_target, hit_ratio, work_ns, l2_resident):
    log2_n = np.atleast_1d(np.asarray(log2_n, dtype=np.float64))
    q = np.zeros(len(log2_n), dtype=QUERY_DTYPE)
    q["log2_n"] = log2_n
    q["fpr_target"] = fpr_target
    q["hit_ratio"] = hit_ratio
    q["work_ns"] = work_ns
    q["l2_resident"] = np.asarray(l2_resident).astype(np.uint32)
    return q


def sample_queries(count, seed):
    """Uniform over log2 n, log10 FPR target, hit ratio and log10 work; half
    of the queries L2-resident."""
    rng = np.random.default_rng(seed)
    return make_queries(rng.uniform(*LOG2_N_RANGE, count),
                        10.0 ** rng.uniform(np.log10(FPR_RANGE[0]), np.log10(FPR_RANGE[1]), count),
                        rng.uniform(*HIT_RANGE, count),
                        10.0 ** rng.uniform(np.log10(WORK_NS_RANGE[0]), np.log10(WORK_NS_RANGE[1]), count),
                        rng.random(count) < 0.5)


def feasible_queries(model, count, seed):
    """sample_queries, keeping only queries that some candidate can meet."""
    out, s = [], seed
    while sum(len(o) for o in out) < count:
        q = sample_queries(count, s)
        out.append(q[model.search(q)["best"] >= 0])
        s += 7919
    return np.concatenate(out)[:count]


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class CostModel:
    """Calibration tables + FPR tables for one candidate set."""

    def __init__(self, calib: CalibrationData, l2_budget_bytes=L2_BUDGET_BYTES, bpk_grid=BPK_GRID):
        self.calib = calib
        self.candidates = calib.candidates
        self.bpk = np.ascontiguousarray(bpk_grid, dtype=np.float64)
        self.fpr = np.ascontiguousarray(np.stack([c.fpr(self.bpk) for c in self.candidates]), dtype=np.float64)
        self.ns = np.ascontiguousarray(calib.ns_per_key, dtype=np.float64)
        self.ns_second = (None if calib.ns_second is None
                          else np.ascontiguousarray(calib.ns_second, dtype=np.float64))
        lb = calib.log2_bytes
        step = float(lb[1] - lb[0]) if len(lb) > 1 else 1.0
        if len(lb) > 2 and not np.allclose(np.diff(lb), step, atol=1e-6):
            raise ValueError("calibration sizes must be evenly spaced in log2(bytes)")
        self.l2_budget_bytes = float(l2_budget_bytes)
        self.tables = _lib.CostTablesS(len(self.candidates), len(self.bpk), _ptr(self.bpk), _ptr(self.fpr), len(lb),
                                       float(lb[0]), step, _ptr(self.ns), float(calib.ns_per_match),
                                       self.l2_budget_bytes, _ptr(self.ns_second))

    @property
    def n_cand(self):
        return len(self.candidates)

    def search(self, queries, per_candidate=False, threads=0):
        """Exhaustive search: best candidate, its cost and bits per key (and,
        with per_candidate, every candidate's best cost and bits per key)."""
        q = np.ascontiguousarray(queries, dtype=QUERY_DTYPE)
        n = len(q)
        best = np.empty(n, dtype=np.int32)
        best_cost = np.empty(n)
        best_bpk = np.empty(n)
        cc = np.empty((n, self.n_cand)) if per_candidate else None
        cb = np.empty((n, self.n_cand)) if per_candidate else None
        t0 = time.perf_counter()
        _lib.check(_lib.lib().dtlg_cost_search(C.byref(self.tables), _ptr(q), n, _ptr(cc), _ptr(cb), _ptr(best),
                                               _ptr(best_cost), _ptr(best_bpk), int(threads)), "cost_search")
        out = {"best": best, "best_cost": best_cost, "best_bpk": best_bpk, "seconds": time.perf_counter() - t0}
        if per_candidate:
            out["cand_cost"], out["cand_bpk"] = cc, cb
        return out

    def evaluate(self, queries, cand, bpk_index):
        q = np.ascontiguousarray(queries, dtype=QUERY_DTYPE)
        cand = np.ascontiguousarray(cand, dtype=np.int32)
        k = np.ascontiguousarray(bpk_index, dtype=np.uint32)
        cost = np.empty(len(q))
        _lib.check(_lib.lib().dtlg_cost_eval(C.byref(self.tables), _ptr(q), len(q), _ptr(cand), _ptr(k), _ptr(cost)),
                   "cost_eval")
        return cost

    def bpk_index(self, bits_per_key):
        """Nearest grid index of a bits-per-key value."""
        b = np.nan_to_num(np.asarray(bits_per_key, dtype=np.float64), nan=1.0)
        k = np.rint(np.log2(np.maximum(b, 1.0)) * BPK_STEPS_PER_OCTAVE)
        return np.clip(k, 0, len(self.bpk) - 1).astype(np.int64)

    def repair(self, queries, cand, k):
        """Move a choice of grid index k to the nearest feasible index: up to the
        least bits per key meeting the FPR target, down to the L2 budget.
        Returns (k, feasible)."""
        q = np.asarray(queries)
        k = np.array(k, dtype=np.int64)
        ok = np.zeros(len(q), dtype=bool)
        for i in range(len(q)):
            if cand[i] < 0:
                continue
            f = self.fpr[cand[i]]
            feas = np.nonzero(f <= q["fpr_target"][i])[0]
            if q["l2_resident"][i]:
                nbytes = 2.0 ** q["log2_n"][i] * self.bpk[feas] / 8.0
                feas = feas[nbytes <= self.l2_budget_bytes]
            if len(feas) == 0:
                continue
            ok[i] = True
            if k[i] < feas[0]:
                k[i] = feas[0]
            elif k[i] > feas[-1]:
                k[i] = feas[-1]
            elif not (f[k[i]] <= q["fpr_target"][i]):
                k[i] = feas[np.searchsorted(feas, k[i])]
        return k, ok


class Skyline:
    """The reference's cached search (skyline_matrix.hpp:22-162,
    skyline_matrix_builder.cpp:19-276) over this model's query space: the best
    (configuration, bits per key) at every grid point, looked up by the next
    grid point at or above the query's n and work, at or below its FPR target,
    the nearest hit ratio and the same residency; the bits per key are then
    repaired to meet the query's own FPR target and budget."""

    LOG2_N = np.arange(10, 29, 1.0)
    LOG10_FPR = np.arange(-1.0, -5.01, -1.0)
    HIT = np.array([0.0, 0.3, 0.6, 0.9])
    WORK = 5.0 * 2.0 ** np.arange(0, 8)

    def __init__(self, model: CostModel):
        self.model = model
        g = np.array(np.meshgrid(self.LOG2_N, self.LOG10_FPR, self.HIT, self.WORK, [0, 1], indexing="ij"))
        g = g.reshape(5, -1)
        self.queries = make_queries(g[0], 10.0 ** g[1], g[2], g[3], g[4])
        r = model.search(self.queries)
        shape = (len(self.LOG2_N), len(self.LOG10_FPR), len(self.HIT), len(self.WORK), 2)
        self.best = r["best"].reshape(shape)
        self.bpk = r["best_bpk"].reshape(shape)
        self.build_seconds = r["seconds"]

    def lookup(self, queries):
        q = np.asarray(queries)
        i_n = np.clip(np.searchsorted(self.LOG2_N, q["log2_n"] - 1e-9), 0, len(self.LOG2_N) - 1)
        lf = np.log10(q["fpr_target"])
        i_f = np.clip(np.searchsorted(-self.LOG10_FPR, -lf - 1e-9), 0, len(self.LOG10_FPR) - 1)
        i_h = np.abs(q["hit_ratio"][:, None] - self.HIT[None, :]).argmin(axis=1)
        i_w = np.clip(np.searchsorted(self.WORK, q["work_ns"] - 1e-9), 0, len(self.WORK) - 1)
        i_r = q["l2_resident"].astype(np.int64)
        cand = self.best[i_n, i_f, i_h, i_w, i_r]
        bpk = np.nan_to_num(self.bpk[i_n, i_f, i_h, i_w, i_r], nan=1.0)
        return cand, bpk
