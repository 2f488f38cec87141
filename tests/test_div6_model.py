"""CPU model of the division-free s/6 of the REF and time-variant updates
(div6_rn in meq_common.cuh): q = RN(s RN(1/6)), r = s - 6q (one fma, exact),
q' = RN(q + r RN(1/6)) (one fma) equals the correctly rounded s/6 for every
normal s in [2^-900, 2^1000].  Exact rational arithmetic stands in for the
fma; the GPU test (test_gpu_div6.py) checks the device code itself."""
from fractions import Fraction

import numpy as np

Z = 1.0 / 6.0


def model(s):
    q = s * Z                                   # RN(s z)
    r_exact = Fraction(s) - 6 * Fraction(q)
    r = float(r_exact)                          # fma(-q, 6, s): one rounding
    assert Fraction(r) == r_exact               # ... of an exactly representable value
    return float(Fraction(r) * Fraction(Z) + Fraction(q))  # fma(r, z, q)


def test_model_equals_correctly_rounded_quotient():
    rng = np.random.default_rng(6)
    xs = [float(np.ldexp(1.0 + rng.random(), int(e))) for e in rng.integers(-900, 1000, 20000)]
    # the values the step forms, ((k + 2k) + 2k) + k, and the binade edges
    for k in np.ldexp(rng.random(5000) + 0.5, rng.integers(-890, 10, 5000)):
        k2 = 2.0 * float(k)
        xs.append(((float(k) + k2) + k2) + float(k))
    for e in (-900, -1, 0, 1, 999):
        b = float(np.ldexp(1.0, e))
        xs += [b, float(np.nextafter(b, 0.0)), float(np.nextafter(b, np.inf)), 6.0 * b, 3.0 * b]
    for s in xs:
        for v in (s, -s):
            assert model(v) == v / 6.0, v
