"""Batched parameter sweeps (tasep_batch_*) against the single-system oracle.

Each system of a batch must end where the oracle's classical RK4 from the
same rates ends: probabilities within 1e-12 for a fixed number of steps, and,
under the exit rule, the same exit step (within the rounding-level slack the
single-system tests allow) and the steady state within 1e-12.  Both sweep
schedules are exercised, as is retirement: systems that converge early stop
changing while the rest continue.
"""
import numpy as np
import pytest

import oracle as O
import tasep_b200 as T

pytestmark = pytest.mark.gpu


def sweep_rates(n, nsys, seed):
    rng = np.random.default_rng(seed)
    ab = rng.uniform(0.2, 1.5, (nsys, 2))
    hops = rng.uniform(0.5, 1.5, (nsys, n - 1))
    return np.column_stack([ab[:, 0], hops, ab[:, 1]])


@pytest.mark.parametrize("schedule", [0, 1])
def test_batch_fixed_steps_matches_oracle(schedule):
    n, nsys, steps = 13, 5, 300
    R = sweep_rates(n, nsys, 1)
    with T.Batch(n, nsys) as b:
        b.set_rates(R)
        b.init(T.INIT_EMPTY)
        res, used = b.run(0.01, steps, exit_rule=False, schedule=schedule)
        assert used == schedule
        for s in range(nsys):
            xo, _ = O.run(n, R[s], h=0.01, steps=steps, integrator=O.INT_RK4, init=O.INIT_EMPTY, exit_rule=False)
            assert res[s]["steps_done"] == steps
            assert np.max(np.abs(b.store(s) - xo)) <= 1e-12


def test_batch_each_system_to_its_own_steady_state():
    n, nsys = 12, 8
    R = sweep_rates(n, nsys, 2)
    R[0, 0] = R[0, -1] = 1.5   # fast
    R[1, 0] = R[1, -1] = 0.25  # slow
    with T.Batch(n, nsys) as b:
        b.set_rates(R)
        b.init(T.INIT_EMPTY)
        res, used = b.run(0.01, 400000, stop_tol=1e-10)
        rho = b.densities()
        finals = [b.store(s) for s in range(nsys)]
    steps = [r["steps_done"] for r in res]
    assert all(r["converged"] == 1 for r in res)
    assert steps[1] > steps[0]  # systems retire at different steps
    for s in range(nsys):
        xo, ro = O.run(n, R[s], h=0.01, steps=400000, integrator=O.INT_RK4, init=O.INIT_EMPTY, stop_tol=1e-10)
        assert abs(int(res[s]["steps_done"]) - int(ro["steps_done"])) <= 2
        assert np.max(np.abs(finals[s] - xo)) <= 1e-12
        assert np.allclose(rho[s], O.densities(n, xo), rtol=1e-12, atol=0)


def test_batch_mixed_precision_densities():
    n, nsys = 13, 4
    R = sweep_rates(n, nsys, 3)
    with T.Batch(n, nsys, T.PRECISION_MIXED) as b:
        b.set_rates(R)
        b.init(T.INIT_EMPTY)
        res, _ = b.run(0.01, 400000, stop_tol=1e-10)
        rho = b.densities()
    assert all(r["converged"] == 1 for r in res)
    for s in range(nsys):
        xo, _ = O.run(n, R[s], h=0.01, steps=400000, integrator=O.INT_RK4, init=O.INIT_EMPTY, stop_tol=1e-10)
        assert np.max(np.abs(rho[s] - O.densities(n, xo))) <= 1e-6


# The standard sweep (1024 systems, n = 16, (alpha, beta) grid, seed-2 hops):
# a 32-system slice spread over the grid.
SLICE = [32 * a + b for a in (4, 9, 14, 19) for b in (4, 7, 10, 13, 16, 19, 22, 25)]


def test_sweep_slice_fixed_steps_matches_oracle():
    """32 systems of the standard n = 16 sweep, 300 RK4 steps: every system
    within 1e-12 of the oracle's single-system run."""
    from tasep_b200.sweep import sweep_rates
    R = sweep_rates()[SLICE]
    n, steps = 16, 300
    with T.Batch(n, len(SLICE)) as b:
        b.set_rates(R)
        b.init(T.INIT_EMPTY)
        res, _ = b.run(0.01, steps, exit_rule=False)
        finals = [b.store(s) for s in range(len(SLICE))]
    for s in range(len(SLICE)):
        xo, _ = O.run(n, R[s], h=0.01, steps=steps, integrator=O.INT_RK4, init=O.INIT_EMPTY, exit_rule=False)
        assert res[s]["steps_done"] == steps
        assert np.max(np.abs(finals[s] - xo)) <= 1e-12


def test_sweep_slice_each_system_to_its_own_exit_rule():
    """The same 32 systems under the exit rule: each retires on its own step,
    equal (within the rounding-level slack of the other exit tests) to the
    single-system integrator's run of that rate vector, with the state within
    1e-12; two of them also against the oracle's own run to the exit rule."""
    from tasep_b200.sweep import sweep_rates
    R = sweep_rates()[SLICE]
    n, tol, cap = 16, 1e-8, 400000
    with T.Batch(n, len(SLICE)) as b:
        b.set_rates(R)
        b.init(T.INIT_EMPTY)
        res, _ = b.run(0.01, cap, stop_tol=tol)
        finals = [b.store(s) for s in range(len(SLICE))]
    steps = [r["steps_done"] for r in res]
    assert all(r["converged"] == 1 for r in res)
    assert len(set(steps)) > 8  # systems retire at different steps
    for s in range(len(SLICE)):
        with T.Meq(n, T.INTEGRATOR_RK4) as m:
            m.set_rates(R[s])
            m.init(T.INIT_EMPTY)
            rs = m.run(0.01, cap, stop_tol=tol)
            x = m.store()
        assert abs(int(rs["steps_done"]) - int(steps[s])) <= 2
        assert np.max(np.abs(finals[s] - x)) <= 1e-12
    for s in sorted(range(len(SLICE)), key=lambda k: steps[k])[:2]:
        xo, ro = O.run(n, R[s], h=0.01, steps=cap, integrator=O.INT_RK4, init=O.INIT_EMPTY, stop_tol=tol)
        assert abs(int(ro["steps_done"]) - int(steps[s])) <= 2
        assert np.max(np.abs(finals[s] - xo)) <= 1e-12


def test_autotuner_picks_a_valid_schedule_and_changes_no_result():
    """schedule=-1: the autotuner times the schedules and reports the one it
    kept; results equal those of a fixed schedule bit for bit (a schedule only
    decides which CTA sweeps which tile)."""
    n, nsys, steps = 13, 6, 200
    R = sweep_rates(n, nsys, 4)
    out = {}
    for sched in (-1, 0, 1, 2):
        with T.Batch(n, nsys) as b:
            b.set_rates(R)
            b.init(T.INIT_EMPTY)
            res, used = b.run(0.01, steps, exit_rule=False, schedule=sched)
            out[sched] = (used, [b.store(s) for s in range(nsys)])
            if sched == -1:
                cfg = b.last_config()
    assert out[-1][0] in (0, 1, 2)
    assert cfg[0] == out[-1][0]
    assert cfg[1] == 2048 and cfg[2] == 0  # tile engines: 2^11 states per tile
    with T.Batch(n, nsys) as b:  # the cluster engine's autotuner: a shape that covers the system
        b.set_rates(R)
        b.init(T.INIT_EMPTY)
        b.run(0.01, 20, exit_rule=False, schedule=2)
        sched, spc, ctas = b.last_config()
    assert sched == 2 and spc in (2048, 4096, 8192) and spc * ctas == 1 << n
    for s in range(nsys):
        assert np.array_equal(out[-1][1][s], out[out[-1][0]][1][s])



@pytest.mark.parametrize("n,precision", [(12, T.PRECISION_FP64), (14, T.PRECISION_FP64), (16, T.PRECISION_FP64),
                                         (17, T.PRECISION_FP64), (15, T.PRECISION_MIXED)])
def test_cluster_resident_fixed_steps_matches_oracle(n, precision):
    """Schedule 2 (each system in the shared memory of one cluster, partners in
    other CTAs read through distributed shared memory), fixed steps: FP64
    within 1e-12 of the oracle's single-system RK4, mixed densities within 1e-6."""
    nsys, steps = 5, 150
    R = sweep_rates(n, nsys, 10 + n)
    with T.Batch(n, nsys, precision) as b:
        b.set_rates(R)
        b.init(T.INIT_EMPTY)
        res, used = b.run(0.01, steps, exit_rule=False, schedule=2)
        assert used == 2
        finals = [b.store(s) for s in range(nsys)]
        rho = b.densities()
    for s in range(nsys):
        xo, _ = O.run(n, R[s], h=0.01, steps=steps, integrator=O.INT_RK4, init=O.INIT_EMPTY, exit_rule=False)
        assert res[s]["steps_done"] == steps
        if precision == T.PRECISION_FP64:
            assert np.max(np.abs(finals[s] - xo)) <= 1e-12
        else:
            assert np.max(np.abs(rho[s] - O.densities(n, xo))) <= 1e-6
            assert abs(finals[s].sum() - 1.0) <= 1e-8


def test_cluster_resident_retires_systems_at_their_own_exit():
    """More systems than clusters, each to its own exit rule: the queue hands
    out systems as others converge; every one ends where the single-system
    integrator ends."""
    n, nsys = 13, 40
    R = sweep_rates(n, nsys, 21)
    tol, cap = 1e-7, 200000
    with T.Batch(n, nsys) as b:
        b.set_rates(R)
        b.init(T.INIT_EMPTY)
        res, used = b.run(0.01, cap, stop_tol=tol, schedule=2)
        finals = [b.store(s) for s in range(nsys)]
    assert all(r["converged"] == 1 for r in res)
    for s in range(0, nsys, 5):
        with T.Meq(n, T.INTEGRATOR_RK4) as m:
            m.set_rates(R[s])
            m.init(T.INIT_EMPTY)
            rs = m.run(0.01, cap, stop_tol=tol)
            x = m.store()
        assert abs(int(rs["steps_done"]) - int(res[s]["steps_done"])) <= 2
        assert np.max(np.abs(finals[s] - x)) <= 1e-12
