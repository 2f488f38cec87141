"""The closure hierarchy (tasep_b200/closure.py) against the reference's
mean-field program (src/mf_full.c), on the CPU.

Golden densities come from the stock program itself (tests/golden/mf_full/,
made by tests/golden/make_mf_golden.py), printed with %lf: the restatement must
agree to that precision (half a unit of the sixth decimal).  With the order
equal to the lattice length nothing is closed and the windows are exact
marginals, so the densities must equal those of the master equation's
classical RK4 (the oracle) to rounding.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from tasep_b200 import closure as CL

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mf_full", "cases.json")
CASES = json.load(open(GOLDEN))


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_matches_stock_mf_full(case):
    V = CL.integrate(np.array(case["rates"]), case["order"], case["t"], case["T"], case["s"])
    rho = CL.densities(V)[0]
    assert np.max(np.abs(rho - np.array(case["rho"]))) <= 5.0001e-7


def test_order_equal_to_length_is_the_master_equation():
    n = 6
    rng = np.random.default_rng(4)
    r = np.concatenate([[0.7], rng.uniform(0.5, 1.5, n - 1), [0.4]])
    V = CL.integrate(r, n, 0.0, 2.0, 200)
    xo, _ = O.run(n, r, h=0.01, steps=200, integrator=O.INT_RK4, init=O.INIT_UNIFORM, exit_rule=False)
    assert np.max(np.abs(CL.densities(V)[0] - O.densities(n, xo)[::-1])) < 1e-14
    # nearest-neighbour covariances from the width-2 windows
    cov_me = O.covariance(n, xo, O.densities(n, xo))[0]
    nn = np.array([cov_me[s, s + 1] for s in range(n - 1)])
    assert np.max(np.abs(CL.nn_covariances(V)[0] - nn)) < 1e-14


def test_higher_closures_approach_the_exact_steady_state():
    """Homogeneous hops: the steady densities of closures of order 1..4 get
    closer to the exact matrix-product values as the order grows."""
    from oracle import mpa
    n, a, b = 10, 0.9, 0.9
    exact = np.array(mpa.densities_float(n, a, b))
    r = np.array([a] + [1.0] * (n - 1) + [b])
    err = [np.max(np.abs(CL.steady_profile(r, k, tol=1e-10)[0] - exact)) for k in (1, 2, 3, 4)]
    assert err[3] < err[2] < err[1] < err[0]
    assert err[3] < 0.01


def test_batched_equals_single():
    rng = np.random.default_rng(9)
    R = np.stack([np.concatenate([[rng.uniform(0.1, 1)], rng.uniform(0.5, 1.5, 7), [rng.uniform(0.1, 1)]])
                  for _ in range(3)])
    Vb = CL.integrate(R, 3, 0.0, 1.0, 100)
    for i in range(3):
        Vs = CL.integrate(R[i], 3, 0.0, 1.0, 100)
        for a, s in zip(Vb, Vs):
            assert np.array_equal(a[i], s[0])
