"""Memory-limit runs: mixed precision (FP64 state, FP32 stage vectors) at
n = 30, 32 and 33 with homogeneous hop rate 1.

* n = 30: the mixed integrator against the FP64 one on the same lattice
  (low-density phase alpha=0.3, beta=0.7 and maximal current alpha=beta=0.9),
  1000 steps from the empty lattice: densities within 1e-6, mass within 1e-8.
* n = 32, 33 (85.9 GB and 171.8 GB of state, which only the mixed layout of
  20 B per state fits into one GPU; the reference's unsigned-int loops cannot
  run n >= 32 at all): started from the exact stationary measure of
  alpha + beta = 1 (a Bernoulli product measure of density alpha), the
  integrator must keep every density at alpha; started from the pair-Markov
  measure of the exact matrix-product densities and nearest-neighbour
  covariances (alpha = beta = 0.9), the densities must stay next to the exact
  ones.  Running n = 33 to its steady state takes hours; these checks take
  seconds.
"""
import numpy as np
import pytest

import tasep_b200 as T
from oracle import mpa

pytestmark = pytest.mark.gpu


def homogeneous(n, a, b):
    return np.array([a] + [1.0] * (n - 1) + [b])


@pytest.mark.parametrize("alpha,beta", [(0.3, 0.7), (0.9, 0.9)])
def test_n30_mixed_against_fp64(alpha, beta):
    n, steps = 30, 1000
    out = {}
    for prec in (T.PRECISION_FP64, T.PRECISION_MIXED):
        with T.Meq(n, T.INTEGRATOR_RK4, prec) as m:
            m.set_rates(homogeneous(n, alpha, beta))
            m.init(T.INIT_EMPTY)
            m.run(0.01, steps, exit_rule=False)
            out[prec] = m.observables()
    d = np.max(np.abs(out[T.PRECISION_MIXED]["rho"] - out[T.PRECISION_FP64]["rho"]))
    assert d <= 1e-6
    assert abs(out[T.PRECISION_MIXED]["mass"] - 1.0) <= 1e-8


@pytest.mark.parametrize("n", [32, 33])
def test_product_measure_stays_stationary(n):
    """alpha + beta = 1: the Bernoulli(alpha) product measure is stationary."""
    a, b = 0.3, 0.7
    exact = np.array(mpa.densities_float(n, a, b))
    assert np.max(np.abs(exact - a)) < 1e-15
    with T.Meq(n, T.INTEGRATOR_RK4, T.PRECISION_MIXED) as m:
        m.set_rates(homogeneous(n, a, b))
        T.init_pair_markov(m, np.full(n, a), np.zeros(n - 1))
        res = m.run(0.01, 3, exit_rule=False)
        obs = m.observables()
    assert res["steps_done"] == 3
    assert res["last_checksum"] < 1e-12  # L1 norm of the increment of the last step
    assert np.max(np.abs(obs["rho"] - a)) <= 1e-12
    assert abs(obs["mass"] - 1.0) <= 1e-10


def test_n33_maximal_current_from_matrix_product_start():
    n, a, b = 33, 0.9, 0.9
    rho = np.array(mpa.densities_float(n, a, b))          # site order
    cov = np.array(mpa.covariance(n, a, b))
    nn = np.array([cov[j, j + 1] for j in range(n - 1)])
    with T.Meq(n, T.INTEGRATOR_RK4, T.PRECISION_MIXED) as m:
        m.set_rates(homogeneous(n, a, b))
        T.init_pair_markov(m, rho, nn)
        obs0 = m.observables()
        m.run(0.01, 5, exit_rule=False)
        obs = m.observables()
    # the start reproduces the exact one- and two-site marginals ...
    assert np.max(np.abs(obs0["rho"][::-1] - rho)) <= 1e-12
    # ... and five steps move no density by more than the start's missing
    # higher correlations allow (rates 1, h = 0.01)
    assert np.max(np.abs(obs["rho"][::-1] - rho)) <= 1e-3
    assert abs(obs["mass"] - 1.0) <= 1e-10
