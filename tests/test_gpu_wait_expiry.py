"""Error path of the bounded device waits, without a GPU fault.

Every wait of the generator sweep on an mbarrier is bounded; when one
expires, the kernel flags the error, lets the bulk copies it issued land and
returns, and the host reports TASEP_ERR_TIMEOUT.  The test hook
tasep_test_inject_wait_expiry shortens the limit to 1 ms and makes the first
CTA leave out one partner copy, so a consumer wait runs out (a barrier that
nothing completes).  Afterwards the same handle must integrate normally and
match the oracle: the context and the handle's device state stay usable.
"""
import numpy as np
import pytest

import oracle as O
import tasep_b200 as T

pytestmark = pytest.mark.gpu


def rates_for(n, seed):
    rng = np.random.default_rng(seed)
    r = np.empty(n + 1)
    r[0], r[n] = rng.uniform(0.1, 1.0, 2)
    r[1:n] = np.clip(rng.lognormal(0.0, 0.5, n - 1), 0.1, 5.0)
    return r


@pytest.fixture
def hook_off():
    yield
    T.inject_wait_expiry(0, -1)


@pytest.mark.parametrize("n,integrator,skip", [(13, T.INTEGRATOR_REF, 0), (13, T.INTEGRATOR_RK4, 0),
                                               (22, T.INTEGRATOR_RK4, 5)])
def test_expired_wait_reports_timeout_and_handle_recovers(n, integrator, skip, hook_off):
    r = rates_for(n, 300 + n)
    x0 = np.random.default_rng(n).random(1 << n)
    x0 /= x0.sum()
    with T.Meq(n, integrator) as m:
        m.set_rates(r)
        m.load(x0)
        T.inject_wait_expiry(1_000_000, skip)
        with pytest.raises(T.TasepError) as ei:
            m.run(0.01, 2, exit_rule=False)
        assert ei.value.status == 5  # TASEP_ERR_TIMEOUT
        T.inject_wait_expiry(0, -1)
        m.load(x0)
        res = m.run(0.01, 3, exit_rule=False)
        x = m.store()
    assert res["steps_done"] == 3
    oi = O.INT_REF if integrator == T.INTEGRATOR_REF else O.INT_RK4
    xo = x0.copy()
    for _ in range(3):
        (O.step_ref if oi == O.INT_REF else O.step_rk4)(n, r, 0.01, xo)
    if integrator == T.INTEGRATOR_REF:
        assert np.array_equal(x, xo)
    else:
        assert np.max(np.abs(x - xo)) <= 1e-12


def test_expired_wait_in_device_step_reports_timeout(hook_off):
    import torch
    assert torch.cuda.is_available(), "CUDA device required"
    n = 14
    r = rates_for(n, 7)
    x = torch.from_numpy(np.random.default_rng(3).random(1 << n)).cuda()
    out = torch.empty_like(x)
    T.inject_wait_expiry(1_000_000, 0)
    with pytest.raises(T.TasepError) as ei:
        T.step_ref_device(n, r, 0.01, x.data_ptr(), out.data_ptr())
    assert ei.value.status == 5
    T.inject_wait_expiry(0, -1)
    cs = T.step_ref_device(n, r, 0.01, x.data_ptr(), out.data_ptr())
    xo = x.cpu().numpy().copy()
    cso = O.step_ref(n, r, 0.01, xo)
    assert np.array_equal(out.cpu().numpy(), xo)
    assert cs == pytest.approx(cso, rel=1e-13)
