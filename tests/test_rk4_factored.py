"""The factored form of classical RK4 used by the constant-rate sweeps
(v1 = z x, v2 = (z - r) v1, w = (z + p) v2, x' = x + (z w + q v2) / 24 with
z = hM and 24 Q(z) = z^3 + 4 z^2 + 12 z + 24 = (z - r)(z^2 + p z + q)) is the
classical RK4 step of the oracle up to rounding (CPU, FP64)."""
import numpy as np

import oracle as O


def factors():
    roots = np.roots([1.0, 4.0, 12.0, 24.0])
    r = float(roots[np.argmin(np.abs(roots.imag))].real)
    return r, 4.0 + r, -24.0 / r


def test_factors_reproduce_the_taylor_coefficients():
    r, p, q = factors()
    # (z - r)(z^2 + p z + q) = z^3 + (p - r) z^2 + (q - p r) z - q r
    assert abs((p - r) - 4.0) < 1e-14 and abs((q - p * r) - 12.0) < 1e-13 and abs(-q * r - 24.0) < 1e-13
    assert -3.0 < r < -2.5 and p > 0 and q > 0  # intermediate vectors keep their sign pattern


def test_factored_step_equals_oracle_rk4():
    r, p, q = factors()
    for n, seed in ((6, 1), (9, 2), (12, 3)):
        rng = np.random.default_rng(seed)
        rates = rng.uniform(0.2, 2.0, n + 1)
        x = rng.random(1 << n)
        x /= x.sum()
        h = 0.01
        v1 = h * O.apply(n, rates, x)
        v2 = h * O.apply(n, rates, v1) - r * v1
        w = h * O.apply(n, rates, v2) + p * v2
        xf = x + (h * O.apply(n, rates, w) + q * v2) / 24.0
        xo = x.copy()
        O.step_rk4(n, rates, h, xo)
        assert np.max(np.abs(xf - xo)) <= 1e-16
