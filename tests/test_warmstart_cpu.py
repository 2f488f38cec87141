"""CPU checks of the warm-start pieces: the network oracle's gradient against
finite differences, the pair-Markov measure's marginals, the features and the
target extraction."""
import numpy as np

from oracle import mlp as omlp
from tasep_b200 import warmstart as ws


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(0)
    p = (rng.standard_normal(omlp.NPARAMS) * 0.3).astype(np.float32)
    # bf16-exact parameters, so the perturbed copies round the same way
    p = omlp.to_bf16(p)
    x = rng.standard_normal((20, omlp.IN))
    t = rng.standard_normal((20, omlp.OUT))
    w = (1.0, 3.0)
    _, g = omlp.loss_grad(p, x, t, w)

    def loss_exact(q):  # same network, no weight rounding
        W1, b1, W2, b2, W3, b3, W4, b4 = omlp.unpack(q)
        h = np.tanh(x @ W1.T + b1)
        h = np.tanh(h @ W2.T + b2)
        h = np.tanh(h @ W3.T + b3)
        d = h @ W4.T + b4 - t
        return float((np.asarray(w) * d * d).sum() / len(x))

    for i in rng.choice(omlp.NPARAMS, 40, replace=False):
        e = np.zeros(omlp.NPARAMS)
        e[i] = 1e-6
        fd = (loss_exact(p + e) - loss_exact(p - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3], dtype=np.float32)
    r = omlp.to_bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -6  # tie to even, rounds up
    assert r[3] == -2.5
    assert abs(r[4] - 1e-3) < 1e-3 * 2 ** -8


def test_pair_markov_marginals():
    rng = np.random.default_rng(1)
    n = 9
    rho = rng.uniform(0.1, 0.9, n)
    cov = rng.uniform(-0.02, 0.02, n - 1)
    p = omlp.pair_markov(n, rho, cov)
    assert abs(p.sum() - 1) < 1e-13 and p.min() >= 0
    _, r, c = ws.profile_targets(p, n)
    assert np.abs(r - rho).max() < 1e-13
    assert np.abs(c[: n - 1] - cov).max() < 1e-13


def test_features_and_targets():
    rates = np.arange(1, 12, dtype=np.float64) / 10  # n = 10
    f = ws.site_features(rates)
    mf = ws.mean_field_profile(rates)
    assert f.shape == (10, 16)
    assert np.allclose(f[0, :9], [0, 0, 0, 0, 0.1, 0.2, 0.3, 0.4, 0.5])
    assert np.allclose(f[9, :9], [0.6, 0.7, 0.8, 0.9, 1.0, 1.1, 0, 0, 0])
    assert np.allclose(f[3, 9:11], [1 / 4, 1 / 7])
    assert np.allclose(f[5, 11:13], [0.1, 1.1])
    assert np.allclose(f[5, 13:16], mf[4:7])
    assert np.allclose(f[0, 13], 0) and np.allclose(f[9, 15], 1)
    # a batch gives the rows of the single calls
    R = np.stack([rates, rates[::-1]])
    assert np.array_equal(ws.site_features(R)[1], ws.site_features(rates[::-1]))
    # an empty lattice has zero densities and covariances
    x = np.zeros(1 << 10)
    x[0] = 1
    y, rho, cov = ws.profile_targets(x, 10)
    assert not y.any()


def test_mean_field_profile():
    # homogeneous hops 1 on the line alpha + beta = 1: the mean-field fixed
    # point is the exact flat profile rho = alpha (J = alpha (1 - alpha))
    r = np.array([0.3] + [1.0] * 11 + [0.7])
    assert np.abs(ws.mean_field_profile(r) - 0.3).max() < 1e-9
    # a slow bond in the middle: a jam upstream, depletion downstream
    r = np.array([1.0] + [1.0] * 7 + [0.1] + [1.0] * 7 + [1.0])
    mf = ws.mean_field_profile(r)
    assert mf[:7].mean() > 0.8 and mf[9:].mean() < 0.2


def test_dataset_roundtrip(tmp_path):
    rng = np.random.default_rng(3)
    data = {12: (ws.sample_rates(12, 3, rng), rng.random((3, 12, 2)).astype(np.float32))}
    ws.save_data(tmp_path / "d.npz", data)
    back = ws.load_data(tmp_path / "d.npz")
    assert np.array_equal(back[12][0], data[12][0]) and np.array_equal(back[12][1], data[12][1])
    X, Y = ws.dataset(back)
    assert X.shape == (36, 16) and Y.shape == (36, 2)
    R = ws.sample_rates(20, 100, np.random.default_rng(0))
    assert R.shape == (100, 21)
    assert R[:, [0, 20]].min() >= 0.05 and R[:, [0, 20]].max() <= 1.5
    assert R[:, 1:20].min() >= 0.1 and R[:, 1:20].max() <= 5.0


def test_pair_field_profile():
    from oracle import mpa
    # exact on alpha + beta = 1 (product measure): density alpha, no correlations
    r = np.array([0.3] + [1.0] * 9 + [0.7])
    rho, cov = ws.pair_field_profile(r)
    assert np.abs(rho - 0.3).max() < 1e-9 and np.abs(cov).max() < 1e-9
    # maximal current: closer to the exact densities than first-order mean field,
    # and nearest-neighbour covariances of the right size
    n = 10
    r = np.array([0.9] + [1.0] * (n - 1) + [0.9])
    exact = np.array(mpa.densities_float(n, 0.9, 0.9))
    C = np.array(mpa.covariance(n, 0.9, 0.9))
    rho, cov = ws.pair_field_profile(r)
    assert np.abs(rho - exact).max() < np.abs(ws.mean_field_profile(r) - exact).max()
    assert np.abs(cov - np.diag(C, 1)).max() < 0.02
    # batched rows equal single calls
    R = ws.sample_rates(12, 3, np.random.default_rng(1))
    rb, cb = ws.pair_field_profile(R, max_steps=3000)
    r1, c1 = ws.pair_field_profile(R[2], max_steps=3000)
    assert np.allclose(rb[2], r1) and np.allclose(cb[2], c1)


def test_mean_field_profile_library_equals_numpy_form():
    """The library's mean-field feature performs the numpy form's operations in
    the same order: equal bit for bit, single vectors and batches."""
    rng = np.random.default_rng(11)
    for n in (2, 7, 16, 24):
        R = ws.sample_rates(n, 3, rng)
        assert np.array_equal(ws.mean_field_profile(R), ws._mean_field_profile_numpy(R))
        assert np.array_equal(ws.mean_field_profile(R[1]), ws._mean_field_profile_numpy(R[1]))
