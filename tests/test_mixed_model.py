"""Mixed precision: does a compensated state update matter?  (CPU model.)

The mixed integrator stores the three intermediate vectors of the factored
RK4 step (v1 = z x, v2 = (z - r) v1, w = (z + p) v2 with z = hM) in FP32 and
keeps the state, the increment D = (z w + q v2) / 24 and the update x + D in
FP64.  A
compensated (Kahan) update would also carry the rounding error of x + D from
step to step, at the price of one more vector (4 B per state: n = 33 would no
longer fit in one GPU).  This model of the mixed step (FP64 products rounded
to FP32 wherever the kernels store FP32) runs both updates to the exit rule:
the compensation changes the converged densities by about 2e-12, while the
FP32 stage vectors put both ~1e-9 away from the FP64 integrator, the error
the compensation cannot reach.  The kernels therefore use the plain FP64
update.
"""
import numpy as np

import oracle as O


def rates_for(n, seed):
    rng = np.random.default_rng(seed)
    r = np.empty(n + 1)
    r[0], r[n] = rng.uniform(0.1, 1.0, 2)
    r[1:n] = np.clip(rng.lognormal(0.0, 0.5, n - 1), 0.1, 5.0)
    return r


def mixed_model_run(n, r, h, compensated, max_steps=400000, tol=1e-10, stop_count=100):
    f32 = lambda v: v.astype(np.float32).astype(np.float64)  # noqa: E731
    x = np.zeros(1 << n)
    x[0] = 1.0
    comp = np.zeros(1 << n)
    early = 0
    rr = np.roots([1.0, 4.0, 12.0, 24.0])
    rt = float(rr[np.argmin(np.abs(rr.imag))].real)  # the real root of 24 Q(z)
    p, q = 4.0 + rt, -24.0 / rt
    for i in range(max_steps):
        v1 = f32(h * O.apply(n, r, x))
        v2 = f32(h * O.apply(n, r, v1) - rt * v1)
        w = f32(h * O.apply(n, r, v2) + p * v2)
        D = (h * O.apply(n, r, w) + q * v2) / 24.0
        if compensated:
            y = D - comp
            t = x + y
            comp = f32((t - x) - y)
            x = t
        else:
            x = x + D
        early = early + 1 if np.abs(D).sum() < tol * h else 0
        if early > stop_count:
            return x, i + 1
    return x, max_steps


def test_compensated_update_is_below_the_fp32_stage_error():
    n = 10
    r = rates_for(n, 5)
    xp, sp = mixed_model_run(n, r, 0.01, False)
    xk, sk = mixed_model_run(n, r, 0.01, True)
    x64, ro = O.run(n, r, h=0.01, steps=400000, integrator=O.INT_RK4, init=O.INIT_EMPTY, stop_tol=1e-10)
    rp, rk, r64 = O.densities(n, xp), O.densities(n, xk), O.densities(n, x64)
    assert sp == sk == ro["steps_done"]
    d_comp = np.abs(rp - rk).max()
    d_plain, d_kahan = np.abs(rp - r64).max(), np.abs(rk - r64).max()
    assert d_comp < 1e-11
    assert d_plain < 1e-6 and d_kahan < 1e-6        # the mixed-precision bar
    assert d_comp < 0.01 * d_plain                 # the compensation is noise next to the FP32 error
    assert abs(d_kahan - d_plain) < 0.05 * d_plain  # and does not bring mixed closer to FP64
