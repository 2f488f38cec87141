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


# ---- correlations: the matrix-product ansatz in an explicit representation ----
#
# The reference's two_point_function (src/steadystates_gmp.c:188-326) evaluates
# <tau_i tau_j> from closed-form sums over Catalan-type coefficients.  Here the
# same quantity comes from the ansatz itself: with C = D + E,
#   <tau_i tau_j> = <W| C^i D C^(j-i-1) D C^(n-j-1) |V> / <W| C^n |V>
# (sites 0-based, i < j).  D and E are the standard bidiagonal representation
# of DE = D + E, D|V> = |V>/beta, <W|E = <W|/alpha, scaled so that every entry
# is rational: D = diag(1/beta, 1, 1, ...) + superdiagonal 1; E = diag(1/alpha,
# 1, 1, ...) + subdiagonal (c, 1, 1, ...) with c = 1/alpha + 1/beta -
# 1/(alpha beta); W = V = e_0.  A product of m matrices applied to e_0 reaches
# level m at most, so dimension n + 2 is exact.

def _rep(n: int, alpha: float, beta: float):
    ia, ib = Fraction(1.0 / alpha), Fraction(1.0 / beta)
    c = ia + ib - ia * ib
    dim = n + 2
    D = [[Fraction(0)] * dim for _ in range(dim)]
    E = [[Fraction(0)] * dim for _ in range(dim)]
    for k in range(dim):
        D[k][k] = ib if k == 0 else Fraction(1)
        E[k][k] = ia if k == 0 else Fraction(1)
        if k + 1 < dim:
            D[k][k + 1] = Fraction(1)
            E[k + 1][k] = c if k == 0 else Fraction(1)
    C = [[D[r][k] + E[r][k] for k in range(dim)] for r in range(dim)]
    return D, C


def _row_times(v, M):
    dim = len(v)
    return [sum((v[r] * M[r][k] for r in range(dim) if v[r]), Fraction(0)) for k in range(dim)]


def _word(n, D, C, marks):
    """<W| prod_{s=0..n-1} (D if s in marks else C) |V>."""
    v = [Fraction(0)] * len(D)
    v[0] = Fraction(1)
    for s in range(n):
        v = _row_times(v, D if s in marks else C)
    return v[0]


def densities_ansatz(n: int, alpha: float, beta: float):
    """<tau_j> from the representation (cross-check of densities())."""
    D, C = _rep(n, alpha, beta)
    Z = _word(n, D, C, ())
    return [_word(n, D, C, (j,)) / Z for j in range(n)]


def two_point(n: int, alpha: float, beta: float):
    """Exact <tau_i tau_j> for all site pairs (n x n; the diagonal is <tau_i>)."""
    D, C = _rep(n, alpha, beta)
    Z = _word(n, D, C, ())
    out = [[Fraction(0)] * n for _ in range(n)]
    for i in range(n):
        out[i][i] = _word(n, D, C, (i,)) / Z
        for j in range(i + 1, n):
            out[i][j] = out[j][i] = _word(n, D, C, (i, j)) / Z
    return out


def covariance(n: int, alpha: float, beta: float):
    """Exact connected correlations <tau_i tau_j> - <tau_i><tau_j> (site order), as floats."""
    T = two_point(n, alpha, beta)
    return [[float(T[i][j] - T[i][i] * T[j][j]) for j in range(n)] for i in range(n)]
