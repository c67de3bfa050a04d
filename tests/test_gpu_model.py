"""The MLP cost model's CUDA kernels (csrc/mlp.cu) against the float64 oracle,
and the trained model's choices against the exhaustive search."""
import os

import numpy as np
import pytest

import model_oracle as MO

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from dtlg.model.calibration import DEFAULT_PATH  # noqa: E402
from dtlg.model.mlp import MLP  # noqa: E402
from dtlg.model.planner import DEFAULT_WEIGHTS, Planner, evaluate  # noqa: E402

DIMS = (5, 64, 3, 568)  # n_in, width, hidden layers, n_out of the cost model


def make(seed=0, dims=DIMS, max_batch=1024):
    m = MLP(dims[0], dims[1], dims[2], dims[3], max_batch=max_batch)
    p = m.init_params(seed)
    return m, p.astype(np.float64)


def batch(rng, n, n_in, n_out):
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    t = rng.normal(size=(n, n_out)).astype(np.float32)
    w = (rng.uniform(0, 1, (n, n_out)) * (rng.random((n, n_out)) < 0.7)).astype(np.float32)
    return x, t, w


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n", [1, 37, 1024, 3000])
def test_forward_matches_float64_oracle(n):
    m, p = make(1, max_batch=1024)
    rng = np.random.default_rng(n)
    x, _, _ = batch(rng, n, DIMS[0], DIMS[3])
    y = m.forward(cuda(x)).cpu().numpy()
    want = MO.forward(p, m.dims, x.astype(np.float64))[-1]
    np.testing.assert_allclose(y, want, rtol=1e-4, atol=1e-4 * np.abs(want).max())


@pytest.mark.parametrize("n", [64, 513, 1024])
def test_gradients_match_float64_oracle(n):
    m, p = make(2)
    rng = np.random.default_rng(100 + n)
    x, t, w = batch(rng, n, DIMS[0], DIMS[3])
    loss = m.loss_grad(cuda(x), cuda(t), cuda(w))
    g = m.get_grads().astype(np.float64)
    want_loss, want_g = MO.loss_grad(p, m.dims, x, t, w)
    assert abs(loss - want_loss) <= 1e-5 * abs(want_loss)
    for (gW, gb), (wW, wb) in zip(m.layers(g), m.layers(want_g)):
        assert np.abs(gW - wW).max() <= 2e-5 * max(np.abs(wW).max(), 1e-12)
        assert np.abs(gb - wb).max() <= 2e-5 * max(np.abs(wb).max(), 1e-12)


def test_adam_step_matches_oracle():
    m, p = make(3)
    rng = np.random.default_rng(4)
    x, t, w = batch(rng, 256, DIMS[0], DIMS[3])
    mom, vel = np.zeros_like(p), np.zeros_like(p)
    for step in range(1, 4):
        m.loss_grad(cuda(x), cuda(t), cuda(w))
        g = m.get_grads().astype(np.float64)
        m.adam_step(1e-3)
        p, mom, vel = MO.adam(p, g, mom, vel, step, 1e-3)
        got = m.get_params().astype(np.float64)
        np.testing.assert_allclose(got, p, rtol=1e-5, atol=1e-6)
        p = got  # follow the device trajectory (fp32 rounding)


def test_training_is_deterministic_and_reduces_loss():
    rng = np.random.default_rng(5)
    x, _, w = batch(rng, 4000, DIMS[0], 40)
    t = np.tanh(x @ rng.normal(size=(DIMS[0], 40))).astype(np.float32)   # a learnable target
    rows = cuda(np.concatenate([rng.permutation(4000) for _ in range(20)])[:300 * 256].astype(np.int32))
    params = []
    for _ in range(2):
        m = MLP(DIMS[0], 64, 3, 40, max_batch=1024)
        m.init_params(7)
        curve = m.train(cuda(x), cuda(t), cuda(w), rows, 256, 3e-3, 1e-4).cpu().numpy()
        params.append(m.get_params())
    assert np.array_equal(params[0], params[1])
    assert curve[-20:].mean() < 0.2 * curve[:5].mean()


def test_choose_is_argmin_of_forward():
    m, p = make(6)
    rng = np.random.default_rng(6)
    x, _, _ = batch(rng, 777, DIMS[0], DIMS[3])
    xd = cuda(x)
    y = m.forward(xd).cpu().numpy()
    choice, aux = m.choose(xd, 284)
    choice, aux = choice.cpu().numpy(), aux.cpu().numpy()
    np.testing.assert_array_equal(choice, np.argmin(y[:, :284], axis=1))
    np.testing.assert_array_equal(aux, y[np.arange(777), 284 + choice])


@pytest.mark.skipif(not (os.path.exists(DEFAULT_PATH) and os.path.exists(DEFAULT_WEIGHTS)),
                    reason="no calibration data / trained weights")
def test_trained_model_is_within_5pct_of_exhaustive_search():
    """2000 held-out queries: the MLP's choices against the exhaustive search's
    best total cost, next to the reference's skyline lookup (the method
    without the network) and the best single configuration."""
    planner = Planner.load()
    rep = evaluate(planner)
    assert rep["eval_queries"] == 2000
    mlp, sky = rep["mlp"], rep["skyline"]
    assert mlp["mean_regret"] <= 0.05, rep
    assert mlp["mean_regret"] < sky["mean_regret"], rep
    assert mlp["mean_regret"] < rep["best_fixed_config"]["mean_regret"], rep
    assert rep["exhaustive"]["mean_regret"] == 0.0


@pytest.mark.skipif(not (os.path.exists(DEFAULT_PATH) and os.path.exists(DEFAULT_WEIGHTS)),
                    reason="no calibration data / trained weights")
def test_planner_config_builds_a_filter_meeting_the_target():
    import dtlg
    from dtlg import keygen
    planner = Planner.load()
    n = 1 << 18
    for target in (1e-2, 1e-3):
        cfg, m_bits = planner.config_for(n, target, hit_ratio=0.1, work_ns=50.0)
        f = dtlg.construct(cfg, m_bits)
        data = f.alloc_filter_data()
        assert f.batch_insert(data, keygen.build_keys_torch(n, 3))
        pk, _ = keygen.probe_keys_torch(n, 1 << 22, 0.0, 3)
        pos = torch.empty(pk.numel(), dtype=torch.int32, device="cuda")
        fpr = f.batch_contains(data, pk, pk.numel(), pos, 0) / pk.numel()
        assert fpr <= target * 1.3, (cfg, m_bits, fpr)


@pytest.mark.skipif(not (os.path.exists(DEFAULT_PATH) and os.path.exists(DEFAULT_WEIGHTS)),
                    reason="no calibration data / trained weights")
def test_facade_for_workload_builds_and_probes():
    import dtlg
    from dtlg import keygen
    for method in ("mlp", "skyline", "exhaustive"):
        f = dtlg.filter.for_workload(1 << 16, work_ns=100.0, fpr_target=1e-3, hit_ratio=0.2, method=method)
        f.insert(keygen.build_keys_torch(1 << 16, 4))
        pk, member = keygen.probe_keys_torch(1 << 16, 1 << 18, 0.2, 4)
        pos = torch.empty(pk.numel(), dtype=torch.int32, device="cuda")
        cnt = f.probe()(pk, pos, 0)
        assert cnt >= int(member.sum().item())
