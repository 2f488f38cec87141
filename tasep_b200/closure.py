"""Closure hierarchy of the TASEP mean-field equations, a non-learned warm start.

Restates the model of the reference's mean-field program (src/mf_full.c,
get_change :575-650, get_cl_change :918-980, closure_change :982-1028,
solve_rk4_step :1030-1333, closure set-up in main :2719-2735).  The unknowns
are the marginals of contiguous windows: for each width w = 1..order, start
position j = 0..n-w and pattern k (bit l of k = occupation of position j+l),
V_w[j, k] is the probability that positions j..j+w-1 show pattern k.
Positions count from the exit end: position p is lattice site n-1-p, i.e.
bit p of a master-equation state index (the reference stores the rates
reversed as well: jr[p] = r[n-p], jr[0] = beta, jr[n] = alpha,
src/mf_full.c:2606-2618).

Each window changes through the moves that touch it: the hop into its top
position (entry when the window ends at the entry site), the hop out of its
bottom position (exit when it starts at the exit site) and the hops inside
it.  The boundary hops involve the window one site wider; for w < order that
window is itself an unknown, for w = order it is closed as a Markov chain of
order `order`-1:
    V_(m+1)[j, K] ~ V_m[j, K mod 2^m] * V_m[j+1, K >> 1] / V_(m-1)[j+1, (K >> 1) mod 2^(m-1)]
(order 1: the product of the two single-site marginals), set to 0 when one
of the factors is below 1e-19 (src/mf_full.c:1012-1024).  order = n gives the
exact master-equation marginals (no closure is used).

Integration is the reference's classical RK4 on all windows (stage inputs
orig + h/2 k1, orig + h/2 k2, orig + h k3; update (k1+2k2+2k3+k4)/6;
negative values clamped to 0) from the uniform product measure V_w = 2^-w
(init_state, src/mf_full.c:178-194).  The evaluation order of each window's
right-hand side follows get_change term by term, so results agree with the
reference program to rounding (checked against its output in the tests).

Everything is batched: rates of shape (c, n+1) give arrays of shape
(c, n-w+1, 2^w).  Host-side numpy; the windows of a lattice number
sum_w (n-w+1) 2^w (about 800 for n = 28 and order 4), far below anything
that would pay for a device kernel.
"""
from __future__ import annotations

import numpy as np

CLOSURE_FLOOR = 10e-20  # src/mf_full.c:1012, 1019


def _jr(rates):
    """Reference rate order: jr[p] for p = 0..n, jr[0] = beta, jr[n] = alpha."""
    R = np.atleast_2d(np.asarray(rates, dtype=np.float64))
    return R[:, ::-1].copy()


def initial_windows(c, n, order):
    """Uniform product measure: every window value 2^-w (src/mf_full.c:178-194)."""
    return [np.full((c, n - w + 1, 1 << w), 0.5 ** w) for w in range(1, order + 1)]


def _closed(V, m):
    """Values of the (m+1)-site windows from the m-site ones (closure_change)."""
    Vm = V[m - 1]
    c, nm1, _ = Vm.shape
    K = np.arange(1 << (m + 1))
    jp = np.arange(nm1 - 1)[:, None]
    u0 = Vm[:, jp, (K & ((1 << m) - 1))[None, :]]
    u1 = Vm[:, jp + 1, (K >> 1)[None, :]]
    small = (u0 < CLOSURE_FLOOR) | (u1 < CLOSURE_FLOOR)
    val = u0 * u1
    if m > 1:
        l0 = V[m - 2][:, jp + 1, ((K >> 1) & ((1 << (m - 1)) - 1))[None, :]]
        small |= l0 < CLOSURE_FLOOR
        val = val / np.where(l0 < CLOSURE_FLOOR, 1.0, l0)
    return np.where(small, 0.0, val)


def rhs(V, jr, order):
    """d V_w / dt for w = 1..order (get_change / get_cl_change)."""
    n = jr.shape[1] - 1
    out = []
    for w in range(1, order + 1):
        i = w - 1
        Vw = V[w - 1]
        Vn = V[w] if w < order else (_closed(V, order) if w < n else None)
        nj = n - w + 1
        k = np.arange(1 << w)[None, :]
        j = np.arange(nj)[:, None]
        # top position j+i: hop in from position j+i+1, or entry at the last position
        top = (k >> i) & 1
        tA = np.empty((jr.shape[0], nj, 1 << w))
        if nj > 1:
            KA = np.where(top == 1, k + (1 << i), k + (1 << (i + 1)))
            vA = Vn[:, j[:-1], np.broadcast_to(KA, (nj - 1, 1 << w))]
            tA[:, :-1, :] = np.where(top == 1, 1.0, -1.0) * (jr[:, (j[:-1] + i + 1)] * vA)
        vlast = Vw[:, nj - 1, :]
        KL = np.where(top[0] == 1, k[0] - (1 << i), k[0])
        tA[:, nj - 1, :] = np.where(top[0] == 1, 1.0, -1.0) * (jr[:, n, None] * vlast[:, KL])
        # bottom position j: hop out to position j-1, or exit at position 0
        b0 = k & 1
        tB = np.empty_like(tA)
        if nj > 1:
            KB = np.where(b0 == 1, 2 * k, 2 * (k + 1))
            vB = Vn[:, j[1:] - 1, np.broadcast_to(KB, (nj - 1, 1 << w))]
            tB[:, 1:, :] = np.where(b0 == 1, -1.0, 1.0) * (jr[:, j[1:]] * vB)
        K0 = np.where(b0[0] == 1, k[0], k[0] + 1)
        tB[:, 0, :] = np.where(b0[0] == 1, -1.0, 1.0) * (jr[:, 0, None] * Vw[:, 0, K0])
        ch = tA + tB
        # hops inside the window, ascending
        for l in range(i):
            bl, bl1 = (k >> l) & 1, (k >> (l + 1)) & 1
            gain = (bl == 1) & (bl1 == 0)
            lose = (bl == 0) & (bl1 == 1)
            idx = np.where(gain, k + (1 << l), k)
            r = jr[:, (j + l + 1)]
            g = r * Vw[:, np.broadcast_to(j, (nj, 1 << w)), np.broadcast_to(idx, (nj, 1 << w))]
            ch = ch + np.where(gain, g, 0.0)
            ch = ch - np.where(lose, r * Vw, 0.0)
        out.append(ch)
    return out


def rk4_step(V, jr, h, order):
    """One step of solve_rk4_step (src/mf_full.c:1030-1134)."""
    orig = V
    d = rhs(orig, jr, order)
    k1 = [h * x for x in d]
    d = rhs([o + (h * 0.5) * x for o, x in zip(orig, d)], jr, order)
    k2 = [h * x for x in d]
    d = rhs([o + (h * 0.5) * x for o, x in zip(orig, d)], jr, order)
    k3 = [h * x for x in d]
    d = rhs([o + h * x for o, x in zip(orig, d)], jr, order)
    k4 = [h * x for x in d]
    new = []
    for o, a, b, cc, e in zip(orig, k1, k2, k3, k4):
        v = o + (a + 2 * b + 2 * cc + e) / 6.0
        new.append(np.where(v < 0, 0.0, v))
    return new


def integrate(rates, order, t0, t1, steps):
    """The reference program's run: `steps` RK4 steps of h = (t1 - t0)/steps
    from the uniform product measure.  Returns the window values."""
    jr = _jr(rates)
    n = jr.shape[1] - 1
    if not 1 <= order <= n:
        raise ValueError(f"closure order {order} outside 1..{n}")
    h = (t1 - t0) / float(steps)
    V = initial_windows(jr.shape[0], n, order)
    for _ in range(steps):
        V = rk4_step(V, jr, h, order)
    return V


def densities(V):
    """Site-order densities rho[s] = P(site s occupied), shape (c, n)."""
    return V[0][:, ::-1, 1]


def nn_covariances(V):
    """Site-order <tau_s tau_(s+1)> - rho_s rho_(s+1), shape (c, n-1); zero for
    order 1 (product measure)."""
    rho = densities(V)
    if len(V) < 2:
        return np.zeros((rho.shape[0], rho.shape[1] - 1))
    p11 = V[1][:, ::-1, 3]  # window at position n-2-s covers sites s, s+1
    return p11 - rho[:, :-1] * rho[:, 1:]


def steady_profile(rates, order, h=0.05, tol=1e-9, max_steps=200000, check_every=200):
    """Steady state of the closed hierarchy: RK4 from the uniform product
    measure until the largest window change rate is below `tol`.  Returns
    (densities, nearest-neighbour covariances) in site order, for one rate
    vector or a batch, as warm-start inputs."""
    jr = _jr(rates)
    n = jr.shape[1] - 1
    order = min(order, n)
    h = min(h, 0.5 / float(jr.max()))
    V = initial_windows(jr.shape[0], n, order)
    for it in range(max_steps):
        Vn = rk4_step(V, jr, h, order)
        if it % check_every == check_every - 1:
            rate = max(float(np.max(np.abs(a - b))) for a, b in zip(Vn, V)) / h
            if rate < tol:
                V = Vn
                break
        V = Vn
    rho = np.clip(densities(V), 1e-6, 1.0 - 1e-6)
    cov = nn_covariances(V)
    single = np.ndim(rates) == 1
    return (rho[0], cov[0]) if single else (rho, cov)
