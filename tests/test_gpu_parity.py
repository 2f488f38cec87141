"""GPU parity: the sm_100a kernels against the CPU oracle, through the C ABI.

Tolerances (from the integrator spec): probabilities within 1e-12 absolute,
expectations within 1e-12 relative.  The reference-compatible integrator
(REF) and the generator product are held to bit equality with the oracle,
which is itself bit-equal to the reference's compiled step code
(tests/test_oracle_golden.py).
"""
import numpy as np
import pytest

import oracle as O
import tasep_b200 as T
from oracle import mpa

pytestmark = pytest.mark.gpu

PROB_TOL = 1e-12
EXP_RTOL = 1e-12


def rates_for(n, seed):
    rng = np.random.default_rng(seed)
    r = np.empty(n + 1)
    r[0], r[n] = rng.uniform(0.1, 1.0, 2)
    r[1:n] = np.clip(rng.lognormal(0.0, 0.5, n - 1), 0.1, 5.0)
    return r


def torch_dev():
    import torch
    assert torch.cuda.is_available(), "CUDA device required"
    return torch


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 10, 11, 12, 13, 14, 16, 19])
def test_apply_bit_exact(n):
    torch = torch_dev()
    rng = np.random.default_rng(100 + n)
    r = rates_for(n, n)
    x = rng.random(1 << n)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    T.apply_device(n, r, xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    y = yd.cpu().numpy()
    yo = O.apply(n, r, x)
    assert np.array_equal(y, yo), f"max diff {np.max(np.abs(y - yo))}"
    # generator columns sum to zero: 1^T M x = 0
    assert abs(y.sum()) < 1e-12 * max(1.0, np.abs(y).sum())


@pytest.mark.parametrize("n", [3, 11, 12, 15])
def test_step_ref_device_bit_exact(n):
    torch = torch_dev()
    rng = np.random.default_rng(7 + n)
    r = rates_for(n, 2 * n)
    x = rng.random(1 << n)
    x /= x.sum()
    xd = torch.from_numpy(x).cuda()
    od = torch.empty_like(xd)
    cs = T.step_ref_device(n, r, 0.01, xd.data_ptr(), od.data_ptr())
    xo = x.copy()
    cso = O.step_ref(n, r, 0.01, xo)
    assert np.array_equal(od.cpu().numpy(), xo)
    assert cs == pytest.approx(cso, rel=1e-13)


@pytest.mark.parametrize("n,init", [(4, O.INIT_EMPTY), (6, O.INIT_UNIFORM), (10, O.INIT_EMPTY),
                                    (12, O.INIT_EMPTY), (13, O.INIT_UNIFORM), (14, O.INIT_EMPTY)])
def test_run_ref_matches_oracle(n, init):
    r = rates_for(n, 30 + n)
    steps = 3000 if n <= 12 else 400
    xo, ro = O.run(n, r, h=0.01, steps=steps, init=init, stop_tol=1e-7)
    with T.Meq(n, T.INTEGRATOR_REF) as m:
        m.set_rates(r)
        m.init(init)
        res = m.run(0.01, steps, stop_tol=1e-7)
        x = m.store()
    assert res["steps_done"] == ro["steps_done"]
    assert res["early_stop"] == ro["early_stop"]
    assert np.array_equal(x, xo), f"max diff {np.max(np.abs(x - xo))}"
    assert res["last_checksum"] == pytest.approx(ro["last_checksum"], rel=1e-12)


def test_run_ref_converges_like_reference_config1():
    """n=10, alpha=.6, beta=.4, gamma=1, uniform start, coded 1e-7 rule:
    the reference converges after step 20935 (exit on the 101st qualifying step)."""
    n = 10
    r = np.array([0.6] + [1.0] * 9 + [0.4])
    xo, ro = O.run(n, r, h=0.01, steps=30000, init=O.INIT_UNIFORM, stop_tol=1e-7)
    with T.Meq(n, T.INTEGRATOR_REF) as m:
        m.set_rates(r)
        m.init(T.INIT_UNIFORM)
        res = m.run(0.01, 30000, stop_tol=1e-7)
        x = m.store()
    assert ro["steps_at_stop"] == 20935
    assert res["steps_at_stop"] == 20935 and res["steps_done"] == 20936
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("n", [5, 10, 12, 14, 16])
def test_run_rk4_fp64(n):
    r = rates_for(n, 50 + n)
    steps = 600
    xo, ro = O.run(n, r, h=0.01, steps=steps, integrator=O.INT_RK4, init=O.INIT_EMPTY, exit_rule=False)
    with T.Meq(n, T.INTEGRATOR_RK4) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res = m.run(0.01, steps, exit_rule=False)
        x = m.store()
        obs = m.observables()
    assert res["steps_done"] == steps
    assert np.max(np.abs(x - xo)) <= PROB_TOL
    yo = O.densities(n, xo)
    assert np.allclose(obs["rho"], yo, rtol=EXP_RTOL, atol=0)
    assert res["last_checksum"] == pytest.approx(ro["last_checksum"], rel=1e-9)


@pytest.mark.parametrize("n", [8, 13])
def test_run_rk4_to_steady_state_exit_rule(n):
    r = rates_for(n, 70 + n)
    xo, ro = O.run(n, r, h=0.01, steps=200000, integrator=O.INT_RK4, init=O.INIT_EMPTY, stop_tol=1e-10)
    with T.Meq(n, T.INTEGRATOR_RK4) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res = m.run(0.01, 200000, stop_tol=1e-10)
        x = m.store()
    assert ro["early_stop"] == 101 and res["converged"] == 1
    assert abs(int(res["steps_done"]) - int(ro["steps_done"])) <= 2
    assert np.max(np.abs(x - xo)) <= 1e-12


@pytest.mark.parametrize("n,integrator", [(6, O.INT_REF), (6, O.INT_RK4), (13, O.INT_REF), (13, O.INT_RK4)])
def test_timevar(n, integrator):
    rng = np.random.default_rng(5)
    base = rates_for(n, 90 + n)
    tv = {"type": rng.integers(0, 3, n + 1), "amplitude": 0.5 * base, "period": rng.uniform(0.5, 2, n + 1),
          "offset": rng.uniform(0, 1, n + 1), "constant": base}
    steps = 500
    xo, ro = O.run(n, base, h=0.01, steps=steps, integrator=integrator, init=O.INIT_EMPTY, timevar=tv,
                   exit_rule=False)
    with T.Meq(n, integrator) as m:
        m.set_rates(base)
        m.set_timevar(tv["type"], tv["amplitude"], tv["period"], tv["offset"], tv["constant"])
        m.init(T.INIT_EMPTY)
        res = m.run(0.01, steps, exit_rule=False)
        x = m.store()
    assert res["steps_done"] == steps
    assert np.max(np.abs(x - xo)) <= PROB_TOL


@pytest.mark.parametrize("n", [9, 14])
def test_mixed_precision_steady_state(n):
    r = rates_for(n, 110 + n)
    xo, ro = O.run(n, r, h=0.01, steps=200000, integrator=O.INT_RK4, init=O.INIT_EMPTY, stop_tol=1e-10)
    with T.Meq(n, T.INTEGRATOR_RK4, T.PRECISION_MIXED) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res = m.run(0.01, 200000, stop_tol=1e-10)
        obs = m.observables()
    assert res["converged"] == 1
    yo = O.densities(n, xo)
    assert np.max(np.abs(obs["rho"] - yo)) <= 1e-6
    # float stage vectors do not sum to zero exactly; the drift stays far below
    # the 1e-6 density bound
    assert abs(obs["mass"] - 1.0) <= 1e-8


@pytest.mark.parametrize("alpha,beta", [(0.3, 0.7), (0.9, 0.9), (0.2, 0.25)])
@pytest.mark.parametrize("precision", [T.PRECISION_FP64, T.PRECISION_MIXED])
def test_homogeneous_steady_state_matches_matrix_product(alpha, beta, precision):
    """Homogeneous hop rates 1: the converged profile against the exact
    matrix-product stationary densities (low-density, maximal-current and
    coexistence-line cases)."""
    n = 14
    exact = np.array(mpa.densities_float(n, alpha, beta))
    with T.Meq(n, T.INTEGRATOR_RK4, precision) as m:
        m.set_rates([alpha] + [1.0] * (n - 1) + [beta])
        m.init(T.INIT_EMPTY)
        res = m.run(0.01, 1000000, stop_tol=1e-10)
        obs = m.observables()
    rho = obs["rho"][::-1]  # site order
    assert res["converged"] == 1
    assert np.max(np.abs(rho - exact)) <= (1e-8 if precision == T.PRECISION_FP64 else 1e-6)
    # connected correlations against the exact two-point function
    cov_exact = np.array(mpa.covariance(n, alpha, beta))
    assert np.max(np.abs(obs["cov"] - cov_exact)) <= (1e-8 if precision == T.PRECISION_FP64 else 1e-6)


@pytest.mark.parametrize("n", [2, 4, 9, 11, 12, 15, 17])
def test_observables(n):
    rng = np.random.default_rng(n)
    x = rng.random(1 << n)
    x /= x.sum()
    with T.Meq(n, T.INTEGRATOR_REF) as m:
        m.set_rates(rates_for(n, 1))
        m.load(x)
        obs = m.observables()
    yo = O.densities(n, x)
    cov, mul = O.covariance(n, x, yo)
    assert np.allclose(obs["rho"], yo, rtol=EXP_RTOL, atol=0)
    assert np.max(np.abs(obs["cov"] - cov)) <= 1e-13
    assert np.max(np.abs(obs["mul"] - mul)) <= 1e-13
    assert obs["mass"] == pytest.approx(x.sum(), rel=1e-14)
    if n >= 4:
        assert np.max(np.abs(obs["window4"] - O.window4(n, x))) <= 1e-14


def _mismatch_report(y, yo, tile_bits=11):
    bad = np.nonzero(y != yo)[0]
    if bad.size == 0:
        return ""
    tiles = np.unique(bad >> tile_bits)
    return (f"{bad.size} mismatches in {tiles.size} tiles; first states {bad[:8].tolist()}, "
            f"max abs diff {np.max(np.abs(y - yo)):.3e}")


@pytest.mark.parametrize("n", [21, 23])
def test_apply_bit_exact_many_tiles_per_cta(n):
    """2^(n-11) tiles over ~148 CTAs: every stage buffer and ring slot is reused many times."""
    torch = torch_dev()
    rng = np.random.default_rng(200 + n)
    r = rates_for(n, 3 * n)
    x = rng.random(1 << n)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    for _ in range(3):  # repeated launches must agree too
        T.apply_device(n, r, xd.data_ptr(), yd.data_ptr())
        torch.cuda.synchronize()
        y = yd.cpu().numpy()
        yo = O.apply(n, r, x)
        assert np.array_equal(y, yo), _mismatch_report(y, yo)


def test_ref_steps_many_tiles_mass_and_parity():
    n = 22
    r = rates_for(n, 7)
    steps = 6
    xo, ro = O.run(n, r, h=0.01, steps=steps, init=O.INIT_UNIFORM, exit_rule=False)
    with T.Meq(n, T.INTEGRATOR_REF) as m:
        m.set_rates(r)
        m.init(T.INIT_UNIFORM)
        m.run(0.01, steps, exit_rule=False)
        x = m.store()
        mass = m.observables()["mass"]
    assert np.array_equal(x, xo), _mismatch_report(x, xo)
    assert abs(mass - 1.0) < 1e-13


def test_rk4_steps_many_tiles():
    n = 21
    r = rates_for(n, 8)
    steps = 5
    xo, ro = O.run(n, r, h=0.01, steps=steps, integrator=O.INT_RK4, init=O.INIT_UNIFORM, exit_rule=False)
    with T.Meq(n, T.INTEGRATOR_RK4) as m:
        m.set_rates(r)
        m.init(T.INIT_UNIFORM)
        m.run(0.01, steps, exit_rule=False)
        x = m.store()
        mass = m.observables()["mass"]
    assert np.max(np.abs(x - xo)) <= PROB_TOL
    assert abs(mass - 1.0) < 1e-13


@pytest.mark.parametrize("integrator,precision", [(T.INTEGRATOR_RK4, T.PRECISION_FP64),
                                                  (T.INTEGRATOR_REF, T.PRECISION_FP64)])
def test_mass_conservation_n24(integrator, precision):
    """Generator columns sum to zero, so the total probability stays 1 to rounding
    (uniform start, 2^24 states, 8192 tiles: every buffer is reused many times)."""
    n = 24
    with T.Meq(n, integrator, precision) as m:
        m.set_rates(rates_for(n, 1))
        m.init(T.INIT_UNIFORM)
        m.run(0.01, 23, exit_rule=False)
        mass = m.observables()["mass"]
        x = m.store()
    assert abs(mass - 1.0) < 1e-12
    assert abs(x.sum() - 1.0) < 1e-12


@pytest.mark.parametrize("n,integrator", [(26, O.INT_RK4), (26, O.INT_REF), (28, O.INT_RK4), (28, O.INT_REF)])
def test_steps_random_dense_state_full_size(n, integrator):
    """A random dense state at n=26 and at the benchmark size n=28 (up to 131072
    tiles, every shared-memory buffer reused hundreds of times per launch): each
    of two steps within 1e-12 of the oracle for every state (REF: bit-exact)."""
    r = rates_for(n, 1)
    x0 = np.random.default_rng(5).random(1 << n)
    x0 /= x0.sum()
    xo = x0.copy()
    with T.Meq(n, integrator) as m:
        m.set_rates(r)
        m.load(x0)
        for _ in range(2):
            m.run(0.01, 1, exit_rule=False)
            if integrator == O.INT_RK4:
                O.step_rk4(n, r, 0.01, xo)
            else:
                O.step_ref(n, r, 0.01, xo)
            y = m.store()
            if integrator == O.INT_REF:
                assert np.array_equal(y, xo), _mismatch_report(y, xo)
            else:
                assert np.max(np.abs(y - xo)) <= PROB_TOL, _mismatch_report(y, xo)


@pytest.mark.parametrize("n,integrator", [(9, T.INTEGRATOR_REF), (14, T.INTEGRATOR_REF), (14, T.INTEGRATOR_RK4)])
def test_run_snapshots_matches_plain_run(n, integrator):
    """tasep_meq_run_snapshots: the hook sees the state after steps 0, R, 2R, ...
    and the run ends where the plain run ends."""
    r = rates_for(n, 130 + n)
    snaps = []
    with T.Meq(n, integrator) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res = m.run_snapshots(0.01, 450, 100, lambda mm, step, t: snaps.append((step, t, mm.store())))
        x = m.store()
    assert [s for s, _, _ in snaps] == [0, 100, 200, 300, 400]
    assert all(abs(t - 0.01 * (s + 1)) < 1e-12 for s, t, _ in snaps)
    with T.Meq(n, integrator) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res2 = m.run(0.01, 450)
        assert np.array_equal(m.store(), x) and res2 == res
    oi = O.INT_REF if integrator == T.INTEGRATOR_REF else O.INT_RK4
    for step, _, xs in snaps:
        xo, _ = O.run(n, r, h=0.01, steps=step + 1, integrator=oi, init=O.INIT_EMPTY)
        assert np.max(np.abs(xs - xo)) <= (0 if integrator == T.INTEGRATOR_REF else PROB_TOL)


@pytest.mark.parametrize("n", [8, 13])
def test_run_snapshots_stop_at_the_exit_rule(n):
    r = rates_for(n, 150 + n)
    steps = []
    with T.Meq(n, T.INTEGRATOR_REF) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res = m.run_snapshots(0.01, 100000, 7, lambda mm, step, t: steps.append(step), stop_tol=1e-4)
    with T.Meq(n, T.INTEGRATOR_REF) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res2 = m.run(0.01, 100000, stop_tol=1e-4)
    assert res == res2 and res["converged"] == 1
    last = res["steps_done"] - 1
    assert steps == list(range(0, last + 1, 7))


@pytest.mark.parametrize("n,integrator", [(9, T.INTEGRATOR_REF), (14, T.INTEGRATOR_RK4), (21, T.INTEGRATOR_REF),
                                          (21, T.INTEGRATOR_RK4)])
def test_run_stream_matches_run_snapshots(n, integrator):
    """tasep_meq_run_stream: the snapshots streamed to the host while the steps
    go on equal, bit for bit, the state and observables that the stopping
    snapshot loop sees at the same steps, and the run ends in the same state."""
    r = rates_for(n, 170 + n)
    seen, streamed = [], []

    def at_stop(mm, step, t):
        seen.append((step, t, mm.store(), mm.observables()))

    with T.Meq(n, integrator) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res = m.run_snapshots(0.01, 450, 50, at_stop)
        x = m.store()
    with T.Meq(n, integrator) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res2 = m.run_stream(0.01, 450, 50, lambda step, t, obs, probs: streamed.append((step, t, probs, obs)),
                            with_probs=True)
        assert np.array_equal(m.store(), x) and res2 == res
    assert [s[0] for s in streamed] == [s[0] for s in seen] == list(range(0, 450, 50))
    for (s1, t1, x1, o1), (s2, t2, x2, o2) in zip(seen, streamed):
        assert t1 == t2 and np.array_equal(x1, x2)
        for k in ("rho", "cov", "mul", "window4"):
            assert np.array_equal(o1[k], o2[k]), k


@pytest.mark.parametrize("n", [8, 19])
def test_run_stream_stops_at_the_exit_rule(n):
    """The streamed loop reads the exit state one chunk behind the device;
    the steps it runs past the exit are no-ops and their snapshots are not
    delivered."""
    r = rates_for(n, 190 + n)
    a, b = [], []
    with T.Meq(n, T.INTEGRATOR_REF) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res = m.run_snapshots(0.01, 100000, 7, lambda mm, step, t: a.append(step), stop_tol=1e-4)
        x = m.store()
    with T.Meq(n, T.INTEGRATOR_REF) as m:
        m.set_rates(r)
        m.init(T.INIT_EMPTY)
        res2 = m.run_stream(0.01, 100000, 7, lambda step, t, obs, probs: b.append((step, probs)), stop_tol=1e-4)
        assert np.array_equal(m.store(), x)
    assert res == res2 and res["converged"] == 1
    assert [s for s, _ in b] == a == list(range(0, res["steps_done"], 7))
    assert all(p is None for _, p in b)


def test_timevar_rk4_many_tiles_per_cta():
    """Time-variant classical RK4 (stage kernels U1..U4, rates evaluated on the
    device at t, t+h/2, t+h/2, t+h) at n=23: 4096 tiles, every partner ring slot
    reused many times per launch; within 1e-12 of the oracle."""
    n = 23
    rng = np.random.default_rng(23)
    base = rates_for(n, 1)
    tv = {"type": np.zeros(n + 1, dtype=np.int32), "amplitude": 0.5 * base,
          "period": rng.uniform(0.5, 2, n + 1), "offset": np.zeros(n + 1), "constant": base}
    x0 = rng.random(1 << n)
    x0 /= x0.sum()
    steps = 4
    xo, _ = O.run(n, base, h=0.01, steps=steps, integrator=O.INT_RK4, x0=x0, timevar=tv, exit_rule=False)
    with T.Meq(n, T.INTEGRATOR_RK4) as m:
        m.set_rates(base)
        m.set_timevar(tv["type"], tv["amplitude"], tv["period"], tv["offset"], tv["constant"])
        m.load(x0)
        res = m.run(0.01, steps, exit_rule=False)
        x = m.store()
    assert res["steps_done"] == steps
    assert np.max(np.abs(x - xo)) <= PROB_TOL, _mismatch_report(x, xo)


@pytest.mark.parametrize("n", [22, 24])
def test_mixed_precision_against_fp64_many_tiles(n):
    """FP32 stage vectors against the FP64 integrator on the same lattice
    (2^22 and 2^24 states, many tiles per CTA): densities within 1e-6 and
    total probability within 1e-8 after 3000 steps from the empty lattice."""
    r = rates_for(n, 2)
    out = {}
    for prec in (T.PRECISION_FP64, T.PRECISION_MIXED):
        with T.Meq(n, T.INTEGRATOR_RK4, prec) as m:
            m.set_rates(r)
            m.init(T.INIT_EMPTY)
            m.run(0.01, 3000, exit_rule=False)
            out[prec] = m.observables()
    assert np.max(np.abs(out[T.PRECISION_MIXED]["rho"] - out[T.PRECISION_FP64]["rho"])) <= 1e-6
    assert abs(out[T.PRECISION_MIXED]["mass"] - 1.0) <= 1e-8
