"""GPU tests of the learned warm start: the training and inference kernels
against the CPU network oracle, the device pair-Markov measure, and what a
trained network gains over the cold start."""
import numpy as np
import pytest

import tasep_b200 as tb
from oracle import mlp as omlp
from tasep_b200 import warmstart as ws

pytestmark = pytest.mark.gpu


def _params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    m = tb.Mlp(seed=seed)
    p = m.params * scale
    p[omlp.NPARAMS - 2:] = rng.uniform(-0.1, 0.1, 2)  # non-zero output bias
    m.params = p
    return m, p


@pytest.mark.parametrize("count", [1, 127, 128, 129, 1000, 5000])
def test_loss_grad_matches_oracle(count):
    m, p = _params(1)
    rng = np.random.default_rng(count)
    x = rng.standard_normal((count, 16)).astype(np.float32)
    t = rng.standard_normal((count, 2)).astype(np.float32)
    w = (1.0, 2.5)
    loss, g = m.loss_grad(x, t, w)
    lref, gref = omlp.loss_grad(p, x, t, w)
    # same BF16 weights; the GPU's forward GEMMs run on the tensor cores with
    # activations split into two BF16 terms (16 significant bits) and FP32
    # accumulation, the oracle in float64
    assert abs(loss - lref) <= 1e-4 * abs(lref)
    assert np.abs(g - gref).max() <= 1e-4 * np.abs(gref).max()
    m.close()


def test_predict_matches_oracle():
    m, p = _params(2)
    x = np.random.default_rng(5).standard_normal((777, 16)).astype(np.float32)
    y = m.predict(x)
    yref, _ = omlp.forward(p, x)
    assert np.abs(y - yref).max() <= 1e-4 * (1 + np.abs(yref).max())
    m.close()


def test_training_reduces_loss_and_is_deterministic():
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, (6000, 16)).astype(np.float32)
    t = np.column_stack([np.sin(x[:, 0] + x[:, 1]) * 0.5, x[:, 2] * x[:, 3]]).astype(np.float32)
    out = []
    for _ in range(2):
        m = tb.Mlp(seed=11)
        losses = m.train(x, t, epochs=30, batch=512, lr=2e-3, seed=5)
        out.append((losses, m.params))
        m.close()
    (l1, p1), (l2, p2) = out
    assert l1[-1] < 0.1 * l1[0]
    assert np.array_equal(l1, l2) and np.array_equal(p1, p2)


@pytest.mark.parametrize("n", [10, 15])
def test_pair_markov_matches_oracle(n):
    rng = np.random.default_rng(n)
    rho = rng.uniform(0.05, 0.95, n)
    cov = rng.uniform(-0.03, 0.03, n - 1)
    with tb.Meq(n, tb.INTEGRATOR_RK4) as m:
        tb.init_pair_markov(m, rho, cov)
        x = m.store()
    ref = omlp.pair_markov(n, rho, cov)
    assert np.abs(x - ref).max() <= 1e-15
    assert abs(x.sum() - 1) < 1e-12


def test_pair_markov_rejects_infeasible():
    with tb.Meq(8, tb.INTEGRATOR_RK4) as m:
        with pytest.raises(tb.TasepError) as e:
            tb.init_pair_markov(m, np.array([0.5] * 7 + [1.0]), np.zeros(7))
        assert e.value.status == 1
        with pytest.raises(tb.TasepError):
            tb.init_pair_markov(m, np.array([0.5] * 3 + [-0.2] + [0.5] * 4), np.zeros(7))


def test_learned_start_gains_over_cold_and_meanfield_starts():
    """Train on batched steady states at n=12 and n=13, then start held-out
    n=14 systems from the prediction.  Every start reaches the empty-lattice
    run's steady state; the learned start needs fewer RK4 steps than the empty
    lattice, and its predicted profile is closer to the steady state than the
    mean-field profile the network is given as input."""
    data, info = ws.generate([(12, 1500), (13, 1000)], seed=3, max_steps=60000)
    assert all(r["converged"] > 0.9 * r["systems"] for r in info)
    X, Y = ws.dataset(data)
    m = tb.Mlp(seed=0)
    losses = ws.train(m, X, Y, schedule=((30, 3e-3), (15, 1e-3)))
    assert losses[-1] < 0.3 * losses[0]
    rows = ws.evaluate(m, 14, 4, seed=4)
    m.close()
    print(ws.summarize(rows))
    for r in rows:
        assert r["empty"]["converged"] and r["learned"]["start"] == "learned"
        for s in ("meanfield", "learned"):
            assert r[s]["converged"] and r[s]["max_density_diff"] < 1e-8
    assert sum(r["learned"]["steps"] for r in rows) < sum(r["empty"]["steps"] for r in rows)
    assert np.median([r["prediction_density_err"] for r in rows]) < np.median(
        [r["meanfield_density_err"] for r in rows])


def test_shipped_network_cuts_wall_time_to_the_exit_rule():
    """The network shipped with the package (trained on n = 12..20) on held-out
    rate vectors at n = 16: the measured wall time to the exit rule, network,
    pair-Markov measure and run included, is at least 1.08x shorter than from
    the empty lattice in total (1.20x measured on 64 vectors at n = 20), and
    each run ends at the empty start's steady state."""
    m = ws.pretrained()
    try:
        rows = ws.evaluate(m, 16, 12, seed=4, starts=("empty", "learned"))
    finally:
        m.close()
    print(ws.summarize(rows, starts=("empty", "learned")))
    for r in rows:
        assert r["empty"]["converged"] and r["learned"]["converged"] and r["learned"]["start"] == "learned"
        assert r["learned"]["max_density_diff"] < 1e-7
    empty = sum(r["empty"]["seconds"] for r in rows)
    learned = sum(r["learned"]["seconds"] for r in rows)
    assert empty / learned > 1.08, (empty, learned)
