"""Configuration choice: the MLP cost model, with the exhaustive search as its
fallback and as the measure of its error.

The network reads a query -- log2 n, log10 of the FPR target, the probe hit
ratio, log10 of the downstream work per tuple and the L2-residency flag --
and predicts, for every candidate configuration c, two numbers:

  * y_c = ln(cost_c / cost_best), the candidate's best cost relative to the
    best candidate's, clipped at Y_MAX (infeasible candidates read Y_MAX);
  * z_c = (log2(bpk_c) - 3.5) / 1.2, the candidate's best bits per key.

The planner takes c = argmin y (dtlg_mlp_choose on the GPU), reads z_c for the
size and moves it to the nearest feasible grid point (FPR target and L2 budget
are analytic, so that step needs no search).  Labels come from the
exhaustive search over the calibration tables, which stays the fallback when
no feasible size exists for the chosen candidate.

    python -m dtlg.model.planner train    (GPU: trains, evaluates, writes weights)
"""
import argparse
import json
import os
import time

import numpy as np

from . import cost as CM
from ._torch import torch_mod
from .calibration import DATA_DIR, CalibrationData
from .mlp import MLP

Y_MAX = 1.0
BPK_CENTER, BPK_SCALE = 3.5, 1.2
WIDTH, HIDDEN = 64, 3
DEFAULT_WEIGHTS = os.path.join(DATA_DIR, "mlp_b200.npz")
TRAIN_QUERIES, EVAL_QUERIES = 60000, 2000
TRAIN_SEED, EVAL_SEED = 11, 999


def features(q):
    """Normalised MLP inputs [N x 5] (float32)."""
    q = np.asarray(q)
    x = np.stack([(q["log2_n"] - 19.0) / 5.2,
                  (np.log10(q["fpr_target"]) + 3.0) / 1.15,
                  (q["hit_ratio"] - 0.45) / 0.26,
                  (np.log10(q["work_ns"]) - 1.7) / 0.58,
                  q["l2_resident"].astype(np.float64) - 0.5], axis=1)
    return np.ascontiguousarray(x, dtype=np.float32)


def targets(search_out, n_cand):
    """Training targets and weights [N x 2C] from a per-candidate search."""
    cc, cb, best = search_out["cand_cost"], search_out["cand_bpk"], search_out["best_cost"]
    with np.errstate(divide="ignore", invalid="ignore"):
        y = np.log(cc / best[:, None])
    y = np.where(np.isfinite(y), y, Y_MAX)
    near = y < Y_MAX
    t = np.zeros((len(cc), 2 * n_cand), dtype=np.float32)
    w = np.zeros_like(t)
    t[:, :n_cand] = np.minimum(y, Y_MAX)
    w[:, :n_cand] = np.where(near, 1.0, 0.05)
    z = (np.log2(np.where(np.isfinite(cb), cb, 2.0 ** BPK_CENTER)) - BPK_CENTER) / BPK_SCALE
    t[:, n_cand:] = z
    w[:, n_cand:] = np.where(y < 0.1, 0.5, 0.0)
    return t, w


class Planner:
    def __init__(self, model: CM.CostModel, mlp: MLP = None):
        self.model = model
        self.mlp = mlp
        self._skyline = None

    @staticmethod
    def load(calibration=None, weights=DEFAULT_WEIGHTS):
        model = CM.CostModel(CalibrationData.load(calibration) if calibration else CalibrationData.load())
        mlp = None
        if weights and os.path.exists(weights):
            z = np.load(weights)
            dims = [int(d) for d in z["dims"]]
            mlp = MLP(dims[0], dims[1], len(dims) - 2, dims[-1])
            mlp.set_params(z["params"])
        return Planner(model, mlp)

    def skyline(self):
        if self._skyline is None:
            self._skyline = CM.Skyline(self.model)
        return self._skyline

    def choose(self, queries, method="mlp"):
        """(candidate index, bits-per-key grid index, cost, used-fallback) per query."""
        q = np.ascontiguousarray(queries, dtype=CM.QUERY_DTYPE)
        m = self.model
        t0 = time.perf_counter()
        if method == "exhaustive":
            r = m.search(q)
            cand, k = r["best"], m.bpk_index(r["best_bpk"])
            fallback = np.zeros(len(q), dtype=bool)
        else:
            if method == "mlp":
                if self.mlp is None:
                    raise RuntimeError("no trained MLP weights")
                torch = torch_mod()
                x = torch.from_numpy(features(q)).cuda()
                choice, aux = self.mlp.choose(x, m.n_cand)
                cand = choice.cpu().numpy().astype(np.int64)
                bpk = 2.0 ** (aux.cpu().numpy().astype(np.float64) * BPK_SCALE + BPK_CENTER)
            elif method == "skyline":
                cand, bpk = self.skyline().lookup(q)
            else:
                raise ValueError(method)
            k, ok = m.repair(q, cand, m.bpk_index(bpk))
            fallback = ~ok
            if fallback.any():  # the exhaustive search stays the fallback
                r = m.search(q[fallback])
                cand = np.array(cand, copy=True)
                cand[fallback] = r["best"]
                k[fallback] = m.bpk_index(r["best_bpk"])
        seconds = time.perf_counter() - t0
        cost = m.evaluate(q, cand, k)
        return {"cand": np.asarray(cand), "bpk_index": k, "cost": cost, "fallback": fallback, "seconds": seconds}

    def config_for(self, n, fpr_target, hit_ratio=0.0, work_ns=50.0, l2_resident=False, method="mlp"):
        """(config, m_bits) for one query: what filter(n, ...) constructs."""
        q = CM.make_queries(np.log2(max(1, n)), fpr_target, hit_ratio, work_ns, l2_resident)
        r = self.choose(q, method)
        c = self.model.candidates[int(r["cand"][0])]
        m_bits = int(np.ceil(n * self.model.bpk[int(r["bpk_index"][0])]))
        return c.config(), uncorrelated_bits(c, m_bits)


def uncorrelated_bits(cand, m_bits):
    """The smallest size >= m_bits whose block (bucket) count has at most one
    factor of two, or is a power of two.

    With MAGIC addressing the block is h0 mod d, h0 = key * C[0] mod 2^32; if
    d = 2^j * d', keys of one block share their low j bits, so the low bits
    of every other multiplicative hash key * C[i] repeat within the block and
    the in-block draws taken from them stop varying: measured with the
    reference's own code path (u64 w=8 s=8 k=8, 2^22 keys, 12 bits per key) the
    FPR is 1.0x the analytic value at 2^0..2^2 factors, 1.5x at 2^3, 1.9x at
    2^7, 2.9x at 2^9 and 11x at 2^15 (d = 3 * 2^15).  The same holds for cuckoo
    bucket counts.  POW2 addressing (the top bits of h0) is not affected."""
    from .. import construct
    blk_bits = cand.block_bytes * 8 if cand.kind == "bloom" else cand.t * cand.b
    blocks = max(1, -(-int(m_bits) // blk_bits))
    for _ in range(1 << 16):
        m = blocks * blk_bits
        f = construct(cand.config(), m)
        bc = f.block_cnt()
        if not f.is_magic() or (bc & 3) != 0:
            return m
        blocks += 1
    return blocks * blk_bits


_SHARED = None


def shared_planner():
    """One Planner per process over the packaged calibration data and weights."""
    global _SHARED
    if _SHARED is None:
        _SHARED = Planner.load()
    return _SHARED


def regret_report(planner, queries, best_cost, methods=("mlp", "skyline", "exhaustive")):
    out = {}
    for meth in methods:
        if meth == "mlp" and planner.mlp is None:
            continue
        r = planner.choose(queries, meth)
        reg = r["cost"] / best_cost - 1.0
        out[meth] = {"mean_regret": float(np.mean(reg)), "median_regret": float(np.median(reg)),
                     "p95_regret": float(np.percentile(reg, 95)), "max_regret": float(np.max(reg)),
                     "within_5pct": float(np.mean(reg <= 0.05)), "fallbacks": int(r["fallback"].sum()),
                     "seconds": r["seconds"]}
    return out


def train(model, n_train=TRAIN_QUERIES, steps=30000, batch=1024, lr_start=2e-3, lr_end=2e-5, seed=0,
          log=print):
    """Labels by the exhaustive search, then Adam on the GPU (dtlg_mlp_train)."""
    torch = torch_mod()
    t0 = time.time()
    q = CM.feasible_queries(model, n_train, TRAIN_SEED)
    r = model.search(q, per_candidate=True)
    t, w = targets(r, model.n_cand)
    x = features(q)
    log(f"labelled {len(q)} training queries by exhaustive search in {time.time() - t0:.1f} s")
    mlp = MLP(x.shape[1], WIDTH, HIDDEN, t.shape[1], max_batch=max(batch, 4096))
    mlp.init_params(seed)
    rng = np.random.default_rng(seed + 1)
    epochs = -(-steps * batch // len(q))
    rows = np.concatenate([rng.permutation(len(q)) for _ in range(epochs)])[:steps * batch].astype(np.int32)
    dx, dt, dw = (torch.from_numpy(a).cuda() for a in (x, t, w))
    drows = torch.from_numpy(rows).cuda()
    torch.cuda.synchronize()
    t1 = time.time()
    curve = mlp.train(dx, dt, dw, drows, batch, lr_start, lr_end)
    torch.cuda.synchronize()
    train_s = time.time() - t1
    curve = curve.cpu().numpy()
    log(f"trained {steps} steps x {batch} rows on the GPU in {train_s:.1f} s; loss {curve[0]:.4f} -> "
        f"{curve[-100:].mean():.5f}")
    info = {"train_queries": len(q), "steps": steps, "batch": batch, "lr": [lr_start, lr_end], "seed": seed,
            "train_seconds": round(train_s, 2), "loss_first": float(curve[0]),
            "loss_last100": float(curve[-100:].mean()), "loss_curve_every_1000": curve[::1000].tolist()}
    return mlp, info


def evaluate(planner, n_eval=EVAL_QUERIES, seed=EVAL_SEED):
    q = CM.feasible_queries(planner.model, n_eval, seed)
    r = planner.model.search(q)
    rep = regret_report(planner, q, r["best_cost"])
    # the best single configuration, sized per query by the search
    rr = planner.model.search(q, per_candidate=True)
    with np.errstate(invalid="ignore"):
        fixed_reg = rr["cand_cost"] / r["best_cost"][:, None] - 1.0
    feasible = np.isfinite(fixed_reg)
    fixed_mean = np.where(feasible, fixed_reg, 0.0).sum(axis=0) / np.maximum(feasible.sum(axis=0), 1)
    fixed_mean[feasible.mean(axis=0) < 0.9] = np.inf   # a fixed choice must serve 90 % of the queries
    bi = int(np.argmin(fixed_mean))
    rep["best_fixed_config"] = {"config": planner.model.candidates[bi].name, "mean_regret": float(fixed_mean[bi]),
                                "feasible": float(feasible[:, bi].mean())}
    rep["eval_queries"] = len(q)
    rep["exhaustive_seconds_per_query"] = r["seconds"] / len(q)
    if planner.mlp is not None:
        torch = torch_mod()
        x = torch.from_numpy(features(q)).cuda()
        planner.mlp.choose(x, planner.model.n_cand)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(10):
            planner.mlp.choose(x, planner.model.n_cand)
        b.record()
        torch.cuda.synchronize()
        rep["mlp_gpu_seconds_per_query"] = a.elapsed_time(b) / 10 / 1e3 / len(q)
    return rep


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--calibration", default=None)
    ap.add_argument("--weights", default=DEFAULT_WEIGHTS)
    ap.add_argument("--steps", type=int, default=30000)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--train-queries", type=int, default=TRAIN_QUERIES)
    ap.add_argument("--report", default=None)
    args = ap.parse_args()
    if args.cmd == "train":
        model = CM.CostModel(CalibrationData.load(args.calibration) if args.calibration else CalibrationData.load())
        mlp, info = train(model, args.train_queries, args.steps, args.batch, args.lr)
        np.savez_compressed(args.weights, params=mlp.get_params(), dims=np.array(mlp.dims),
                            info=json.dumps(info))
        planner = Planner(model, mlp)
    else:
        planner = Planner.load(args.calibration, args.weights)
        info = {}
    rep = evaluate(planner)
    rep["training"] = info
    text = json.dumps(rep, indent=1)
    print(text)
    if args.report:
        with open(args.report, "w") as f:
            f.write(text + "\n")


if __name__ == "__main__":
    main()
