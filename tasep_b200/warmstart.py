"""Learned warm start for the master-equation integrator.

A per-site network (tasep_mlp_* in libtasep_cuda.so) maps the rates around a
site to that site's steady-state density and nearest-neighbour covariance.
It is trained on steady states that the batched master-equation solver
(tasep_batch_*) produces.  Its prediction becomes a pair-Markov initial
measure over all 2^n states, built on the device
(tasep_meq_init_pair_markov), and RK4 runs from there under the usual exit
rule.  The empty lattice remains the fallback when a prediction is infeasible
and the check of the converged result.

Inputs of the network (16 per site j of a lattice of n sites, rates r[0..n],
r[0] = alpha the entry rate, r[i] the hop rate from site i-1 to i, r[n] =
beta the exit rate):
  * the 9 rates r[j-4..j+4] (0 outside 0..n);
  * the distances to both ends as 1/(j+1) and 1/(n-j);
  * alpha and beta;
  * the mean-field densities of sites j-1, j, j+1 (0 left of the lattice, 1
    right of it).
A window of rates cannot see a bottleneck outside it, yet the slowest bond
decides whether a site sits in a jam (upstream) or a depleted stretch
(downstream).  The mean-field profile (mean_field_profile: the current
J_i = r_i rho_(i-1) (1 - rho_i) relaxed to a constant) carries that global
information cheaply; the network corrects it towards the master equation's
profile.  The mean-field profile alone, as a product measure, is also the
non-learned start the learned one is compared with.

Outputs: rho_j and COV_SCALE * (<tau_j tau_(j+1)> - rho_j rho_(j+1)) (0 for
the last site).
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import Batch, INIT_EMPTY, INTEGRATOR_RK4, Meq, Mlp, PRECISION_FP64, TasepError, init_pair_markov, lib
from . import closure

COV_SCALE = 10.0
MF_STEPS = 20000
# parameters trained by `python -m tasep_b200.warmstart` with its defaults:
# 19,992 converged steady states at n = 12..20 (seed 3), 100 epochs
PRETRAINED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_params.npy")


def pretrained(device=-1):
    """The shipped trained network on `device`."""
    m = Mlp(seed=0, device=device)
    m.params = np.load(PRETRAINED)
    return m


def mean_field_profile(rates, steps=MF_STEPS):
    """Mean-field densities for one rate vector (n+1,) or a batch (count, n+1).

    Explicit Euler on d rho_i/dt = J_i - J_(i+1) with J_0 = alpha (1 - rho_0),
    J_i = r_i rho_(i-1) (1 - rho_i), J_n = beta rho_(n-1), from rho = 1/2, with
    dt = 1/(4 max rate) for a fixed number of steps (deterministic; the slow
    modes of long lattices are not fully relaxed, which does not matter for a
    feature).  Computed by tasep_mean_field_profile in the library (the same
    operations in the same order as _mean_field_profile_numpy, bit for bit,
    about 100x faster)."""
    R = np.ascontiguousarray(np.atleast_2d(np.asarray(rates, dtype=np.float64)))
    c, n1 = R.shape
    n = n1 - 1
    rho = np.empty((c, n))
    L = lib()
    L.tasep_mean_field_profile.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    st = L.tasep_mean_field_profile(n, c, int(steps), R.ctypes.data_as(C.POINTER(C.c_double)),
                                    rho.ctypes.data_as(C.POINTER(C.c_double)))
    if st != 0:
        raise TasepError(st, L.tasep_last_error().decode())
    return rho[0] if np.ndim(rates) == 1 else rho


def _mean_field_profile_numpy(rates, steps=MF_STEPS):
    """The same iteration in numpy (the form the network was trained with)."""
    R = np.atleast_2d(np.asarray(rates, dtype=np.float64))
    c, n1 = R.shape
    n = n1 - 1
    dt = 0.25 / R.max(axis=1, keepdims=True)
    rho = np.full((c, n), 0.5)
    J = np.empty((c, n + 1))
    for _ in range(steps):
        J[:, 0] = R[:, 0] * (1.0 - rho[:, 0])
        J[:, 1:n] = R[:, 1:n] * rho[:, :-1] * (1.0 - rho[:, 1:])
        J[:, n] = R[:, n] * rho[:, -1]
        rho += dt * (J[:, :-1] - J[:, 1:])
    rho = np.clip(rho, 1e-6, 1.0 - 1e-6)
    return rho[0] if np.ndim(rates) == 1 else rho


def pair_field_profile(rates, max_steps=MF_STEPS, tol=1e-11):
    """Pair approximation of the steady state: nearest-neighbour pair
    probabilities p_i(a, b) = P(tau_i = a, tau_(i+1) = b) evolved under the
    TASEP moves that change them, with three-site probabilities closed as
    P(a, b, c) = p_(i-1)(a, b) p_i(b, c) / P(tau_i = b) (the first closure of
    the reference's mean-field hierarchy, src/mf_full.c).  Explicit Euler from
    the uniform product measure, dt = 1/(4 max rate), until the largest change
    rate falls below `tol` or `max_steps`.  Returns (densities (n,), nearest-
    neighbour covariances (n-1,)) for one rate vector, or batched arrays."""
    R = np.atleast_2d(np.asarray(rates, dtype=np.float64))
    c, n1 = R.shape
    n = n1 - 1
    dt = 0.25 / R.max(axis=1)[:, None, None, None]
    P = np.full((c, n - 1, 2, 2), 0.25)
    rho = np.empty((c, n))
    tiny = 1e-300
    for it in range(max_steps):
        rho[:, :n - 1] = P[:, :, 1, 0] + P[:, :, 1, 1]
        rho[:, n - 1] = P[:, -1, 0, 1] + P[:, -1, 1, 1]
        d = np.zeros_like(P)
        f = R[:, 1:n] * P[:, :, 1, 0]  # hop inside pair i: site i -> i+1
        d[:, :, 1, 0] -= f
        d[:, :, 0, 1] += f
        gain = np.empty((c, n - 1, 2))  # left site of pair i fills: entry, or hop from site i-1
        gain[:, 0, :] = R[:, 0, None] * P[:, 0, 0, :]
        lose = np.empty((c, n - 1, 2))  # right site of pair i empties: exit, or hop to site i+2
        lose[:, -1, :] = R[:, n, None] * P[:, -1, :, 1]
        if n > 2:
            q0 = np.maximum(1.0 - rho[:, 1:n - 1], tiny)
            gain[:, 1:, :] = R[:, 1:n - 1, None] * P[:, :-1, 1, 0][..., None] * P[:, 1:, 0, :] / q0[..., None]
            q1 = np.maximum(rho[:, 1:n - 1], tiny)
            lose[:, :-1, :] = R[:, 2:n, None] * P[:, :-1, :, 1] * (P[:, 1:, 1, 0] / q1)[..., None]
        d[:, :, 0, :] -= gain
        d[:, :, 1, :] += gain
        d[:, :, :, 1] -= lose
        d[:, :, :, 0] += lose
        P += dt * d
        if it % 500 == 499 and np.abs(d).max() < tol:
            break
    rho[:, :n - 1] = P[:, :, 1, 0] + P[:, :, 1, 1]
    rho[:, n - 1] = P[:, -1, 0, 1] + P[:, -1, 1, 1]
    rho = np.clip(rho, 1e-6, 1.0 - 1e-6)
    cov = P[:, :, 1, 1] - rho[:, :-1] * rho[:, 1:]
    return (rho[0], cov[0]) if np.ndim(rates) == 1 else (rho, cov)


def site_features(rates, mf=None):
    """(n, 16) network inputs of one rate vector, or (count, n, 16) of a batch."""
    R = np.atleast_2d(np.asarray(rates, dtype=np.float64))
    c, n1 = R.shape
    n = n1 - 1
    rho = np.atleast_2d(mean_field_profile(R) if mf is None else mf)
    pad = np.concatenate([np.zeros((c, 4)), R, np.zeros((c, 4))], axis=1)
    rp = np.concatenate([np.zeros((c, 1)), rho, np.ones((c, 1))], axis=1)
    f = np.empty((c, n, 16), dtype=np.float32)
    for j in range(n):
        f[:, j, :9] = pad[:, j:j + 9]  # r[j-4] .. r[j+4]
        f[:, j, 9] = 1.0 / (j + 1)
        f[:, j, 10] = 1.0 / (n - j)
        f[:, j, 11] = R[:, 0]
        f[:, j, 12] = R[:, n]
        f[:, j, 13:16] = rp[:, j:j + 3]  # mean-field rho_(j-1), rho_j, rho_(j+1)
    return f[0] if np.ndim(rates) == 1 else f


def profile_targets(x, n):
    """(n, 2) targets from a state vector: rho_j and COV_SCALE * nearest-neighbour
    covariance (site j is bit n-1-j of the state index, so site 0 is the top bit)."""
    x = np.asarray(x, dtype=np.float64)
    rho = np.array([x.reshape(1 << j, 2, -1)[:, 1, :].sum() for j in range(n)])
    cov = np.zeros(n)
    for j in range(n - 1):
        cov[j] = x.reshape(1 << j, 2, 2, -1)[:, 1, 1, :].sum() - rho[j] * rho[j + 1]
    return np.column_stack([rho, COV_SCALE * cov]).astype(np.float32), rho, cov


def sample_rates(n, count, rng):
    """alpha, beta ~ U[0.05, 1.5]; hops lognormal(0, 0.5) clipped to [0.1, 5]."""
    ab = rng.uniform(0.05, 1.5, (count, 2))
    hops = np.clip(rng.lognormal(0.0, 0.5, (count, n - 1)), 0.1, 5.0)
    return np.column_stack([ab[:, 0], hops, ab[:, 1]])


def generate(sizes, seed=3, h=0.04, stop_tol=1e-7, max_steps=100000, precision=PRECISION_FP64, log=None):
    """Steady states from batched solves.  `sizes` is a list of (n, systems).
    Returns {n: (rates (k, n+1), targets (k, n, 2))} over the systems that met
    the exit rule, and a list of per-size records.  The training targets need
    about 1e-5 accuracy, so the sweep runs with a longer step and a looser exit
    threshold than the integration it seeds."""
    rng = np.random.default_rng(seed)
    data, info = {}, []
    for n, count in sizes:
        R = sample_rates(n, count, rng)
        t0 = time.time()
        with Batch(n, count, precision) as b:
            b.set_rates(R)
            b.init(INIT_EMPTY)
            res, sched = b.run(h, max_steps, stop_tol=stop_tol)
            t_run = time.time() - t0
            keep = [s for s in range(count) if res[s]["converged"]]
            Y = np.stack([profile_targets(b.store(s), n)[0] for s in keep]) if keep else np.zeros((0, n, 2))
        data[n] = (R[keep], Y)
        steps = np.array([r["steps_done"] for r in res])
        info.append({"n": n, "systems": count, "converged": len(keep), "run_seconds": round(t_run, 2),
                     "seconds": round(time.time() - t0, 2), "schedule": sched, "steps_min": int(steps.min()),
                     "steps_median": int(np.median(steps)), "steps_max": int(steps.max())})
        if log:
            log(info[-1])
    return data, info


def dataset(data, ns=None):
    """Per-site training arrays (X (m, 16), Y (m, 2)) from generate()'s output."""
    xs, ys = [], []
    for n, (R, Y) in sorted(data.items()):
        if (ns is not None and n not in ns) or len(R) == 0:
            continue
        xs.append(site_features(R).reshape(-1, 16))
        ys.append(np.asarray(Y, dtype=np.float32).reshape(-1, 2))
    return np.concatenate(xs), np.concatenate(ys)


def save_data(path, data):
    np.savez_compressed(path, **{f"R{n}": R for n, (R, _) in data.items()},
                        **{f"Y{n}": Y for n, (_, Y) in data.items()})


def load_data(path):
    z = np.load(path)
    return {int(k[1:]): (z[k], z["Y" + k[1:]]) for k in z.files if k.startswith("R")}


def predict_profile(mlp, rates):
    y = mlp.predict(site_features(rates))
    n = len(rates) - 1
    rho = y[:, 0].astype(np.float64)
    cov = y[:, 1].astype(np.float64) / COV_SCALE
    return rho, cov[: max(n - 1, 0)]


STARTS = ("empty", "uniform", "meanfield", "pairfield", "closure3", "closure4", "learned", "exactpair")
CLOSURE_TOL = 1e-7  # window change rate at which the closure hierarchy counts as stationary


def closure_start_profile(rates, order):
    """Densities and nearest-neighbour covariances of the steady state of the
    mean-field closure hierarchy of order `order` (tasep_b200/closure.py, the
    reference's src/mf_full.c model) for one rate vector or a batch."""
    return closure.steady_profile(rates, order, tol=CLOSURE_TOL)


def run_to_steady_state(n, rates, start, mlp=None, h=0.01, max_steps=2000000, stop_tol=1e-10, device=-1,
                        profile=None):
    """Classical RK4 (FP64) from `start` to the exit rule: 'empty' (the
    empty lattice), 'uniform' (every state 2^-n), 'meanfield' (product
    measure of the mean-field profile), 'pairfield' (pair-Markov measure of
    the pair approximation), 'learned' (pair-Markov measure of the network's
    prediction) or 'exactpair' (pair-Markov measure of a given profile
    (densities, nearest-neighbour covariances), e.g. the converged one: the
    best any pair-Markov start can do), 'closure3' / 'closure4' (pair-Markov
    measure of the steady state of the mean-field closure hierarchy of that
    order; `profile` may hold it precomputed).  Returns (final state, run result, seconds
    from the start's set-up - profile computation, network inference and
    measure construction included - to the end of the run, the start
    actually used)."""
    m = Meq(n, INTEGRATOR_RK4, PRECISION_FP64, device=device)
    try:
        m.set_rates(rates)
        m.synchronize()
        t0 = time.perf_counter()
        used = start
        if start == "learned":
            rho, cov = predict_profile(mlp, rates)
            try:
                init_pair_markov(m, rho, cov)
            except TasepError:
                m.init(INIT_EMPTY)  # infeasible prediction: cold start
                used = "empty (fallback)"
        elif start == "meanfield":
            init_pair_markov(m, mean_field_profile(rates), np.zeros(n - 1))
        elif start == "pairfield":
            init_pair_markov(m, *pair_field_profile(rates))
        elif start in ("closure3", "closure4"):
            if profile is not None:  # computed ahead for a whole set (batched), time added by the caller
                init_pair_markov(m, profile[0], profile[1][: n - 1])
            else:
                init_pair_markov(m, *closure_start_profile(rates, int(start[-1])))
        elif start == "exactpair":
            init_pair_markov(m, profile[0], profile[1][: n - 1])
        elif start == "uniform":
            init_pair_markov(m, np.full(n, 0.5), np.zeros(n - 1))
        elif start == "empty":
            m.init(INIT_EMPTY)
        else:
            raise ValueError(f"unknown start {start!r}")
        res = m.run(h, max_steps, stop_tol=stop_tol)
        seconds = time.perf_counter() - t0
        return m.store(), res, seconds, used
    finally:
        m.close()


def train(mlp, X, Y, schedule=((50, 3e-3), (30, 1e-3), (20, 3e-4)), batch=512, seed=0, out_weights=(1.0, 1.0)):
    """Mini-batch Adam in phases of (epochs, learning rate); returns the per-epoch losses."""
    losses = []
    for k, (epochs, lr) in enumerate(schedule):
        losses.extend(mlp.train(X, Y, out_weights, epochs=epochs, batch=batch, lr=lr, seed=seed + k).tolist())
    return losses


def evaluate(mlp, n, count, seed=4, h=0.01, max_steps=2000000, starts=("empty", "meanfield", "learned"), log=None):
    """Held-out rate vectors (a seed the training data did not use): every
    start in `starts` run to the exit rule; wall time, steps and the final
    profile's difference from the empty-lattice run, the reference result for the others."""
    assert starts[0] == "empty"
    R = sample_rates(n, count, np.random.default_rng(seed))
    # closure profiles of the whole set in one batched host computation; each
    # system's start is charged its share of that time
    cl_prof, cl_sec = {}, {}
    for s in starts:
        if s in ("closure3", "closure4"):
            t0 = time.perf_counter()
            cl_prof[s] = closure_start_profile(R, int(s[-1]))
            cl_sec[s] = (time.perf_counter() - t0) / len(R)
    rows = []
    for i, r in enumerate(R):
        row = {"n": n, "system": i}
        ref = None
        for s in starts:
            prof = (cl_prof[s][0][i], cl_prof[s][1][i]) if s in cl_prof else ref
            x, res, sec, used = run_to_steady_state(n, r, s, mlp, h=h, max_steps=max_steps, profile=prof)
            sec += cl_sec.get(s, 0.0)
            _, rho, cov = profile_targets(x, n)
            del x
            if ref is None:
                ref = (rho, cov)
            row[s] = {"start": used, "seconds": round(sec, 4), "steps": int(res["steps_done"]),
                      "converged": bool(res["converged"]),
                      "max_density_diff": float(np.abs(rho - ref[0]).max()),
                      "max_cov_diff": float(np.abs(cov - ref[1]).max())}
        rho_p, cov_p = predict_profile(mlp, r)
        row["prediction_density_err"] = float(np.abs(rho_p - ref[0]).max())
        row["prediction_cov_err"] = float(np.abs(cov_p - ref[1][: n - 1]).max())
        row["meanfield_density_err"] = float(np.abs(mean_field_profile(r) - ref[0]).max())
        row["pairfield_density_err"] = float(np.abs(pair_field_profile(r)[0] - ref[0]).max())
        for s in cl_prof:
            row[f"{s}_density_err"] = float(np.abs(cl_prof[s][0][i] - ref[0]).max())
        for s in starts[1:]:
            row[s]["speedup"] = round(row["empty"]["seconds"] / row[s]["seconds"], 3)
        rows.append(row)
        if log:
            log(row)
    return rows


def start_profiles(mlp, R, start, ref_profiles=None):
    """Per-system (densities, nearest-neighbour covariances) of a start for a
    batch of rate vectors R, or None for the empty lattice."""
    n = R.shape[1] - 1
    if start == "empty":
        return None
    if start == "meanfield":
        return [(mean_field_profile(r), np.zeros(n - 1)) for r in R]
    if start == "pairfield":
        rho, cov = pair_field_profile(R)
        return list(zip(rho, cov))
    if start in ("closure3", "closure4"):
        rho, cov = closure_start_profile(R, int(start[-1]))
        return list(zip(rho, cov))
    if start == "learned":
        return [predict_profile(mlp, r) for r in R]
    if start == "exactpair":
        return [(p[0], p[1][: n - 1]) for p in ref_profiles]
    raise ValueError(f"unknown start {start!r}")


def evaluate_batched(mlp, n, count, seed=4, h=0.01, max_steps=4000000, stop_tol=1e-10,
                     starts=("empty", "learned"), device=-1, log=None):
    """The held-out evaluation with all `count` systems of a start in one batch
    (tasep_batch_*), so that 64 vectors at n = 24 fit a GPU session: per system,
    the steps to its exit rule from each start, whose ratio to the empty
    lattice's is the wall-time ratio of single-system runs (every step of a
    system costs the same); the final profile's difference from the
    empty-lattice run; the batch's own wall time.  Starts other than the empty
    lattice are built per system on the device (pair-Markov measure) and loaded
    into the batch; an infeasible profile falls back to the empty lattice."""
    assert starts[0] == "empty"
    R = sample_rates(n, count, np.random.default_rng(seed))
    N = 1 << n
    out = {"n": n, "systems": count, "seed": seed, "h": h, "stop_tol": stop_tol, "starts": {}}
    ref_prof = None
    for st in starts:
        t0 = time.perf_counter()
        prof = start_profiles(mlp, R, st, ref_prof)
        t_prof = time.perf_counter() - t0
        with Batch(n, count, PRECISION_FP64, device=device) as b:
            b.set_rates(R)
            used = [st] * count
            t1 = time.perf_counter()
            if prof is None:
                b.init(INIT_EMPTY)
            else:
                X = np.empty((count, N))
                m = Meq(n, INTEGRATOR_RK4, PRECISION_FP64, device=device)
                try:
                    for s in range(count):
                        m.set_rates(R[s])
                        try:
                            init_pair_markov(m, prof[s][0], prof[s][1])
                        except TasepError:
                            m.init(INIT_EMPTY)
                            used[s] = "empty (fallback)"
                        m.store(X[s])
                finally:
                    m.close()
                b.load(X)
                del X
            t_init = time.perf_counter() - t1
            t2 = time.perf_counter()
            res, sched = b.run(h, max_steps, stop_tol=stop_tol)
            t_run = time.perf_counter() - t2
            finals = [profile_targets(b.store(s), n)[1:] for s in range(count)]
        if st == "empty":
            ref_prof = finals
        rec = {"profile_seconds": round(t_prof, 3), "init_seconds": round(t_init, 3),
               "run_seconds": round(t_run, 3), "schedule": sched,
               "steps": [int(r["steps_done"]) for r in res], "converged": [bool(r["converged"]) for r in res],
               "fallbacks": sum(u != st for u in used),
               "max_density_diff": [float(np.abs(f[0] - rf[0]).max()) for f, rf in zip(finals, ref_prof)],
               "max_cov_diff": [float(np.abs(f[1] - rf[1]).max()) for f, rf in zip(finals, ref_prof)]}
        if prof is not None:
            rec["start_density_err"] = [float(np.abs(p[0] - rf[0]).max()) for p, rf in zip(prof, ref_prof)]
        if st != "empty":
            e = np.array(out["starts"]["empty"]["steps"], dtype=float)
            w = np.array(rec["steps"], dtype=float)
            ratio = e / w
            rec["step_ratio_total"] = round(float(e.sum() / w.sum()), 4)
            rec["step_ratio_median"] = round(float(np.median(ratio)), 4)
            rec["step_ratio_min_max"] = [round(float(ratio.min()), 4), round(float(ratio.max()), 4)]
        out["starts"][st] = rec
        if log:
            log({"n": n, "start": st, **{k: v for k, v in rec.items() if not isinstance(v, list)}})
    return out


def summarize(rows, starts=("empty", "meanfield", "learned")):
    out = {}
    for n in sorted({r["n"] for r in rows}):
        rs = [r for r in rows if r["n"] == n]
        tc = sum(r["empty"]["seconds"] for r in rs)
        s = {"systems": len(rs), "empty_seconds": round(tc, 3),
             "prediction_density_err_median": float(np.median([r["prediction_density_err"] for r in rs])),
             "meanfield_density_err_median": float(np.median([r["meanfield_density_err"] for r in rs])),
             "pairfield_density_err_median": float(np.median([r["pairfield_density_err"] for r in rs]))}
        for st in ("closure3", "closure4"):
            if f"{st}_density_err" in rs[0]:
                s[f"{st}_density_err_median"] = float(np.median([r[f"{st}_density_err"] for r in rs]))
        for st in starts[1:]:
            tw = sum(r[st]["seconds"] for r in rs)
            s[st] = {"seconds": round(tw, 3), "wall_time_ratio": round(tc / tw, 3),
                     "step_ratio": round(sum(r["empty"]["steps"] for r in rs) / sum(r[st]["steps"] for r in rs), 3),
                     "max_density_diff": max(r[st]["max_density_diff"] for r in rs),
                     "all_converged": all(r[st]["converged"] for r in rs)}
        out[f"n{n}"] = s
    return out


def _pairs(text):
    return [tuple(int(v) for v in item.split(":")) for item in text.split(",") if item]


def main(argv=None):
    import argparse
    import json
    import os

    ap = argparse.ArgumentParser(description="train the warm-start network on batched steady states and "
                                             "compare learned, mean-field and cold starts")
    ap.add_argument("--sizes", default="12:6000,13:4000,14:3500,16:3000,18:2500,20:1000", help="n:systems,...")
    ap.add_argument("--data", default=None, help="dataset .npz (read if present, else generated and written)")
    ap.add_argument("--params", default=None, help="trained parameters .npy (read if present, else trained)")
    ap.add_argument("--eval", default="24:8", help="held-out n:count,...")
    ap.add_argument("--epochs", type=float, default=1.0, help="scale of the default training schedule")
    ap.add_argument("--starts", default="empty,meanfield,learned", help="starts to compare (empty first)")
    ap.add_argument("--out", default=None, help="JSON report")
    ap.add_argument("--batched", action="store_true",
                    help="evaluate each start's held-out systems in one batch (steps to the exit rule per system)")
    a = ap.parse_args(argv)
    starts = tuple(a.starts.split(","))

    def log(rec):
        print(json.dumps(rec), flush=True)

    report = {}
    if a.batched:  # evaluation of the shipped (or given) network only
        mlp = Mlp(seed=0)
        mlp.params = np.load(a.params if a.params else PRETRAINED)
        report["eval_batched"] = [evaluate_batched(mlp, n, count, starts=starts, log=log)
                                  for n, count in _pairs(a.eval)]
        if a.out:
            with open(a.out, "w") as f:
                json.dump(report, f, indent=1)
        mlp.close()
        return
    if a.params and os.path.exists(a.params) and not a.data:  # evaluation of a trained network only
        mlp = Mlp(seed=0)
        mlp.params = np.load(a.params)
        rows = []
        for n, count in _pairs(a.eval):
            rows += evaluate(mlp, n, count, starts=starts, log=log)
        report["eval"] = rows
        report["summary"] = summarize(rows, starts)
        log(report["summary"])
        if a.out:
            with open(a.out, "w") as f:
                json.dump(report, f, indent=1)
        mlp.close()
        return
    if a.data and os.path.exists(a.data):
        data = load_data(a.data)
    else:
        t0 = time.time()
        data, report["generate"] = generate(_pairs(a.sizes), log=log)
        report["generate_seconds"] = round(time.time() - t0, 1)
        if a.data:
            save_data(a.data, data)
    report["steady_states"] = {int(n): int(len(R)) for n, (R, _) in data.items()}
    # hold out every tenth system of each size for the validation loss
    train_d = {n: (R[np.arange(len(R)) % 10 != 0], Y[np.arange(len(R)) % 10 != 0]) for n, (R, Y) in data.items()}
    val_d = {n: (R[::10], Y[::10]) for n, (R, Y) in data.items()}
    t0 = time.time()
    X, Y = dataset(train_d)
    Xv, Yv = dataset(val_d)
    report["feature_seconds"] = round(time.time() - t0, 2)
    mlp = Mlp(seed=0)
    if a.params and os.path.exists(a.params):
        mlp.params = np.load(a.params)
    else:
        sched = [(max(1, int(round(e * a.epochs))), lr) for e, lr in ((50, 3e-3), (30, 1e-3), (20, 3e-4))]
        t0 = time.time()
        losses = train(mlp, X, Y, schedule=sched)
        report["train_seconds"] = round(time.time() - t0, 2)
        report["train_loss_first_last"] = [losses[0], losses[-1]]
        if a.params:
            np.save(a.params, mlp.params)
    report["train_samples"] = int(len(X))
    report["val_loss"] = mlp.loss_grad(Xv, Yv)[0]
    P = mlp.predict(Xv)
    report["val_mean_density_err"] = float(np.abs(P[:, 0] - Yv[:, 0]).mean())
    report["val_max_density_err"] = float(np.abs(P[:, 0] - Yv[:, 0]).max())
    report["val_meanfield_mean_density_err"] = float(np.abs(Xv[:, 14] - Yv[:, 0]).mean())
    log({k: report[k] for k in report if k != "generate"})
    rows = []
    for n, count in _pairs(a.eval):
        rows += evaluate(mlp, n, count, starts=starts, log=log)
    report["eval"] = rows
    report["summary"] = summarize(rows, starts)
    log(report["summary"])
    if a.out:
        with open(a.out, "w") as f:
            json.dump(report, f, indent=1)
    mlp.close()


if __name__ == "__main__":
    main()
