"""The CPU oracle pinned against the reference (no GPU).

* the stock reference binary's output files (tests/golden/stock/, made by
  tests/golden/make_golden.py): probabilities printed with %.20g round-trip
  exactly, so the oracle must reproduce them bit for bit, with the same exit
  step; densities, covariances and window observables agree to the printed
  6 decimals;
* the reference's own step code (oracle/_ref, when built): bit for bit;
* the exact matrix-product steady state (oracle/mpa.py): a converged run.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from oracle import mpa

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_case(name):
    d = os.path.join(GOLD, "stock", name)
    with open(os.path.join(d, "run.json")) as f:
        info = json.load(f)
    return d, info


def parse_probs(path):
    idx, val = [], []
    with open(path) as f:
        for line in f:
            bits, v = line.split()
            idx.append(int(bits, 2))  # site 0 first = most significant bit
            val.append(float(v))
    x = np.empty(len(idx))
    x[np.array(idx)] = val
    return x


def argv_get(argv, flag, cast=str, default=None):
    return cast(argv[argv.index(flag) + 1]) if flag in argv else default


def oracle_for_case(info):
    argv = info["argv"]
    n = argv_get(argv, "-n", int)
    t0, T, steps = argv_get(argv, "-t", float), argv_get(argv, "-T", float), argv_get(argv, "-s", int)
    h = float(np.float64((T - t0) / np.longdouble(steps)))  # (T - t)/((long double) steps), :586
    if "rates.txt" in info:
        r = np.array(info["rates.txt"])
    else:
        a, b, g = argv_get(argv, "--alpha", float), argv_get(argv, "--beta", float), argv_get(argv, "--gamma", float)
        r = np.array([a] + [g] * (n - 1) + [b])
    tv = None
    if "timevar" in info:
        t = info["timevar"]
        tv = {"type": [{"s": 0, "c": 1, "l": 2}[c[0]] for c in t["function-type"]], "amplitude": t["amplitude"],
              "period": t["period"], "offset": t["offset"], "constant": t["constant"]}
    x, res = O.run(n, r, h=h, steps=steps, integrator=O.INT_REF, init=O.INIT_UNIFORM, stop_tol=1e-7,
                   exit_rule=tv is None, t0=t0, timevar=tv)
    return n, x, res


CASES = ["cfg1_f", "n7_rows", "n8_f", "n5_timevar"]


@pytest.mark.parametrize("name", CASES)
def test_probabilities_bit_exact_vs_stock_binary(name):
    d, info = load_case(name)
    assert info["returncode"] == 0
    n, x, res = oracle_for_case(info)
    gold = parse_probs(os.path.join(d, "out"))
    assert np.array_equal(x, gold), f"max diff {np.max(np.abs(x - gold))}"
    if info["convergence_after"] is not None:
        assert res["early_stop"] > 0 and res["steps_at_stop"] == int(info["convergence_after"])
    else:
        assert res["early_stop"] == 0


def test_config1_converges_where_the_reference_does():
    _, info = load_case("cfg1_f")
    assert info["convergence_after"] == "20935"
    assert info["sim_time"] == "209.360000"


def _floats(text):
    return [float(t) for t in text.replace(",", " ").split()]


@pytest.mark.parametrize("name", CASES)
def test_observables_vs_stock_binary(name):
    d, info = load_case(name)
    n, x, _ = oracle_for_case(info)
    y = O.densities(n, x)
    vec = _floats(open(os.path.join(d, "out_exp_values_fin.vec")).read())
    assert np.max(np.abs(np.array(vec) - y[::-1])) <= 5e-7  # site order, %lf
    cov, mul = O.covariance(n, x, y)
    gold_cov = np.array(_floats(open(os.path.join(d, "out_cov.mat")).read())).reshape(n, n)
    assert np.max(np.abs(gold_cov - cov)) <= 5e-7
    dim = 1 << n
    # closures and error guesses: windows of 4 sites (src/masterEquation.c:1452-1496)
    for fname, fn in (("out_closures", O.pf_approx), ("out_error_guess", O.error_guess)):
        vals = [float(line.split()[-1]) for line in open(os.path.join(d, fname))]
        mine = [fn(x, 3, 2, n - 2 - i) for i in range(1, n - 2)]
        assert len(vals) == len(mine) and np.max(np.abs(np.array(vals) - mine)) <= 5e-7
    vals = [float(line.split()[-1]) for line in open(os.path.join(d, "out_high_order_point_fun"))]
    mine = [O.point_func(x, 15, 4, n - 4 - i) for i in range(0, n - 3)]
    assert np.max(np.abs(np.array(vals) - mine)) <= 5e-7
    assert dim == x.size


def test_highcorr_file_holds_the_undefined_return_value():
    """high_order_corr falls off its end (src/masterEquation.c:47-75).  The gcc -O2
    binary prints the value left in the return register, le*(no-le)*re*(no-re),
    not the correlation coefficient; documented as a deviation."""
    d, info = load_case("n8_f")
    n, x, _ = oracle_for_case(info)
    rows = [line.split() for line in open(os.path.join(d, "out_highcorr"))][1:]
    for key, row in enumerate(rows):
        printed = [float(v) for v in row[1:]]
        for i, pv in enumerate(printed, start=1):
            off = n - 2 - i
            le = O.point_func(x, key + 4, 3, off)
            no = O.point_func(x, key, 2, off)
            re_ = O.point_func(x, (key << 1) + 1, 3, off - 1)
            ub = le * (no - le) * re_ * (no - re_)
            assert pv == pytest.approx(ub, rel=2e-3, abs=1e-12)


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("n,init,csr", [(2, 0, True), (5, 1, True), (9, 1, False), (11, 0, True)])
def test_oracle_bit_exact_vs_reference_step_code(n, init, csr):
    r = np.random.default_rng(n).uniform(0.1, 2.0, n + 1)
    x1, r1 = O.run(n, r, h=0.01, steps=700, init=init, stop_tol=1e-7)
    x2, r2 = O.ref_run(n, r, h=0.01, steps=700, init=init, stop_tol=1e-7, use_csr=csr)
    assert np.array_equal(x1, x2)
    assert r1 == r2


@pytest.mark.parametrize("name", ["cfg1_empty", "cfg1_empty_converged", "n9_inhom"])
def test_oracle_vs_reference_harness_fixtures(name):
    z = np.load(os.path.join(GOLD, "harness", name + ".npz"))
    n = int(np.log2(z["x"].size))
    x, res = O.run(n, z["rates"], h=0.01, steps=int(z["steps"]), init=O.INIT_EMPTY, stop_tol=float(z["tol"]))
    assert np.array_equal(x, z["x"])
    assert res["steps_done"] == int(z["steps_done"]) and res["early_stop"] == int(z["early_stop"])


def test_generator_columns_sum_to_zero_and_rows_follow_reference_order():
    n = 6
    r = np.random.default_rng(0).uniform(0.1, 2.0, n + 1)
    M = np.zeros((1 << n, 1 << n))
    for i in range(1 << n):
        cols, vals = O.gen_row(n, i, r)
        # entry (if bit n-1), diagonal, exit (if bit 0 clear), hops ascending
        k = 0
        if (i >> (n - 1)) & 1:
            assert cols[0] == i - (1 << (n - 1)) and vals[0] == r[0]
            k = 1
        assert cols[k] == i and vals[k] <= 0
        M[i, cols] += vals
    assert np.max(np.abs(M.sum(axis=0))) < 1e-14
    y = O.apply(n, r, np.ones(1 << n))
    assert np.allclose(y, M.sum(axis=1), atol=1e-14)


def test_mpa_matches_converged_master_equation():
    with open(os.path.join(GOLD, "mpa.json")) as f:
        cases = json.load(f)
    for c in cases[:3]:
        n, a, b = c["n"], c["alpha"], c["beta"]
        x, res = O.run(n, [a] + [1.0] * (n - 1) + [b], h=0.01, steps=400000, stop_tol=1e-10)
        assert res["early_stop"] > 100
        y = O.densities(n, x)[::-1]  # site order
        assert np.max(np.abs(y - np.array(c["rho"]))) < 2e-9
        assert c["rho"] == pytest.approx(mpa.densities_float(n, a, b), abs=0, rel=0)


def test_mpa_product_measure_line():
    """On alpha + beta = 1 the stationary measure is Bernoulli with density alpha."""
    rho = mpa.densities(8, 0.3, 0.7)
    assert max(abs(float(v) - 0.3) for v in rho) < 1e-15


def test_classical_rk4_is_fourth_order():
    n = 6
    r = np.random.default_rng(3).uniform(0.3, 1.5, n + 1)
    x0 = np.zeros(1 << n)
    x0[0] = 1.0
    errs = []
    for h in (0.2, 0.1, 0.05):
        steps = int(round(2.0 / h))
        x, _ = O.run(n, r, h=h, steps=steps, integrator=O.INT_RK4, x0=x0, exit_rule=False)
        xr, _ = O.run(n, r, h=h / 16, steps=steps * 16, integrator=O.INT_RK4, x0=x0, exit_rule=False)
        errs.append(np.max(np.abs(x - xr)))
    rates_ = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(rates_) > 3.7


def test_mpa_representation_matches_reference_densities():
    """The explicit matrix representation behind mpa.two_point gives the same
    densities as the reference's B-table formula (src/steadystates_gmp.c:142-186)."""
    for n, a, b in [(6, 0.3, 0.5), (8, 0.9, 0.9), (9, 1.2, 0.35), (10, 0.6, 0.4)]:
        d1, d2 = mpa.densities(n, a, b), mpa.densities_ansatz(n, a, b)
        assert max(abs(float((x - y) / x)) for x, y in zip(d1, d2)) < 1e-15


def test_mpa_two_point_matches_converged_master_equation():
    """Exact connected correlations against the oracle's converged RK4 state."""
    for n, a, b in [(8, 0.9, 0.9), (8, 0.3, 0.5), (7, 1.2, 0.35)]:
        x, res = O.run(n, [a] + [1.0] * (n - 1) + [b], h=0.01, steps=400000, integrator=O.INT_RK4,
                       init=O.INIT_EMPTY, stop_tol=1e-10)
        assert res["early_stop"] > 100
        cov, _ = O.covariance(n, x)
        assert np.max(np.abs(cov - np.array(mpa.covariance(n, a, b)))) < 1e-9
    # on alpha + beta = 1 the measure is a product measure: no correlations
    c = np.array(mpa.covariance(8, 0.3, 0.7))
    assert np.max(np.abs(c - np.diag(np.diag(c)))) < 1e-15
