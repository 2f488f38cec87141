"""Exact steady state of the open TASEP with hop rate 1 (matrix-product ansatz).

TEST INFRASTRUCTURE ONLY.  Exact-rational restatement of the reference's
``src/steadystates_gmp.c`` (which uses GMP ``mpf`` floats of 64 bits by
default, ``src/steadystates_gmp.c:363``).  ``fractions.Fraction`` replaces
``mpf_t``; the inputs 1/alpha and 1/beta enter as the double values the
reference passes to ``mpf_set_d`` (``src/steadystates_gmp.c:118-119, 166``),
so the only difference from the reference is that no rounding happens after
that point.  Valid only for homogeneous interior hop rate 1.

GMP itself (the third-party arithmetic the reference links with ``-lgmp``,
reference Makefile:50; version unpinned there, libgmp.so.10.5 at run time)
is not needed: exact rationals are a strict refinement of its arithmetic.
"""
from __future__ import annotations

from fractions import Fraction


def eval_B(n: int, p: int) -> Fraction:
    """B(n, p): src/steadystates_gmp.c:20-65."""
    d = n - p
    if d == 0:
        return Fraction(1)
    if d == 1:
        return Fraction(n - 1)
    num, den = 1, 1
    for k in range(d - 1):
        num *= n + d - 1 - k
        den *= d - k
    return Fraction(num * p, den)


def table_B(n: int):
    """B[i][k], i < n, 0 <= k <= n: src/steadystates_gmp.c:68-95."""
    return [[eval_B(i + 1, k) if 0 < k <= i + 1 else Fraction(0) for k in range(n + 1)]
            for i in range(n)]


def table_Z(B, n: int, alpha: float, beta: float):
    """Z[0..n]: src/steadystates_gmp.c:97-140."""
    ia, ib = Fraction(1.0 / alpha), Fraction(1.0 / beta)
    Z = [Fraction(0)] * (n + 1)
    for i in range(n):
        acc = Fraction(0)
        for p in range(i + 2):
            for q in range(p + 1):
                acc += ia ** q * ib ** (p - q) * B[i][p]
        Z[i + 1] = acc
    Z[0] = Fraction(1)
    return Z


def densities(n: int, alpha: float, beta: float):
    """Exact <tau_j>, j = 0 (entry site) .. n-1: src/steadystates_gmp.c:142-186."""
    B = table_B(n)
    Z = table_Z(B, n, alpha, beta)
    ib = Fraction(1.0 / beta)
    rho = []
    for i in range(n - 1):
        acc = Fraction(0)
        for k in range(n - i - 1):
            acc += B[k][1] * Z[n - 1 - k]
            acc += ib ** (k + 2) * B[n - i - 2][k + 1] * Z[i]
        rho.append(acc / Z[n])
    rho.append(Z[n - 1] / (Fraction(beta) * Z[n]))
    return rho


def densities_float(n: int, alpha: float, beta: float):
    return [float(v) for v in densities(n, alpha, beta)]
