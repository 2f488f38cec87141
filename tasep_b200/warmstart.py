"""Learned warm start for the master-equation integrator.

A per-site network (tasep_mlp_* in libtasep_cuda.so) maps the rates around a
site to that site's steady-state density and nearest-neighbour covariance.
It is trained on steady states that the batched master-equation solver
(tasep_batch_*) produces.  Its prediction becomes a pair-Markov initial
measure over all 2^n states, built on the device
(tasep_meq_init_pair_markov), and RK4 runs from there under the usual exit
rule.  The empty lattice remains the fallback when a prediction is infeasible
and the check of the converged result.

Inputs of the network (16 per site j of a lattice of n sites, rates r[0..n]):
the 9 rates r[j-4..j+4] (0 outside 0..n), 1/(j+1) and 1/(n-j), the boundary
rates alpha = r[0] and beta = r[n], the smallest and the mean hop rate, and
n/32.  A window of 9 rates alone cannot see the boundary rates that set the
phase of sites far from the ends, hence the global terms.  Outputs: rho_j and
10 * (<tau_j tau_(j+1)> - rho_j rho_(j+1)) (0 for the last site).
"""
from __future__ import annotations

import time

import numpy as np

from . import Batch, INIT_EMPTY, INTEGRATOR_RK4, Meq, Mlp, PRECISION_FP64, TasepError, init_pair_markov

COV_SCALE = 10.0


def site_features(rates):
    r = np.asarray(rates, dtype=np.float64)
    n = len(r) - 1
    pad = np.concatenate([np.zeros(4), r, np.zeros(4)])
    hops = r[1:n] if n > 1 else np.array([1.0])
    glob = [r[0], r[n], hops.min(), hops.mean(), n / 32.0]
    f = np.empty((n, 16), dtype=np.float32)
    for j in range(n):
        f[j, :9] = pad[j:j + 9]  # r[j-4] .. r[j+4]
        f[j, 9] = 1.0 / (j + 1)
        f[j, 10] = 1.0 / (n - j)
        f[j, 11:] = glob
    return f


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
        if ns is not None and n not in ns:
            continue
        for r, y in zip(R, Y):
            xs.append(site_features(r))
            ys.append(y)
    return np.concatenate(xs), np.concatenate(ys).astype(np.float32)


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


def run_to_steady_state(n, rates, start, mlp=None, h=0.01, max_steps=2000000, stop_tol=1e-10, device=-1):
    """Classical RK4 (FP64) from `start` ('empty', 'uniform' or 'learned') to the
    exit rule.  Returns (final state, run result, seconds from the start's
    set-up - network inference and measure construction included - to the
    end of the run, the start actually used)."""
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
        elif start == "uniform":
            init_pair_markov(m, np.full(n, 0.5), np.zeros(n - 1))
        else:
            m.init(INIT_EMPTY)
        res = m.run(h, max_steps, stop_tol=stop_tol)
        seconds = time.perf_counter() - t0
        return m.store(), res, seconds, used
    finally:
        m.close()


def train(mlp, X, Y, schedule=((60, 1e-3), (40, 3e-4), (30, 1e-4)), batch=1024, seed=0, out_weights=(1.0, 1.0)):
    """Mini-batch Adam in phases of (epochs, learning rate); returns the per-epoch losses."""
    losses = []
    for k, (epochs, lr) in enumerate(schedule):
        losses.extend(mlp.train(X, Y, out_weights, epochs=epochs, batch=batch, lr=lr, seed=seed + k).tolist())
    return losses


def evaluate(mlp, n, count, seed=4, h=0.01, max_steps=2000000, log=None):
    """Held-out rate vectors (a seed the training data did not use): cold and
    learned starts to the exit rule, wall time and final profile difference."""
    R = sample_rates(n, count, np.random.default_rng(seed))
    rows = []
    for i, r in enumerate(R):
        xc, rc, tc, _ = run_to_steady_state(n, r, "empty", h=h, max_steps=max_steps)
        _, rho_c, cov_c = profile_targets(xc, n)
        del xc
        rho_p, cov_p = predict_profile(mlp, r)
        xw, rw, tw, used = run_to_steady_state(n, r, "learned", mlp, h=h, max_steps=max_steps)
        _, rho_w, cov_w = profile_targets(xw, n)
        del xw
        rows.append({"n": n, "system": i, "start": used, "cold_seconds": round(tc, 4), "warm_seconds": round(tw, 4),
                     "cold_steps": int(rc["steps_done"]), "warm_steps": int(rw["steps_done"]),
                     "cold_converged": bool(rc["converged"]), "warm_converged": bool(rw["converged"]),
                     "speedup": round(tc / tw, 3),
                     "max_density_diff": float(np.abs(rho_c - rho_w).max()),
                     "max_cov_diff": float(np.abs(cov_c - cov_w).max()),
                     "prediction_density_err": float(np.abs(rho_p - rho_c).max()),
                     "prediction_cov_err": float(np.abs(cov_p - cov_c[: n - 1]).max())})
        if log:
            log(rows[-1])
    return rows


def _pairs(text):
    return [tuple(int(v) for v in item.split(":")) for item in text.split(",") if item]


def main(argv=None):
    import argparse
    import json
    import os

    ap = argparse.ArgumentParser(description="train the warm-start network on batched steady states and "
                                             "compare learned and cold starts")
    ap.add_argument("--sizes", default="12:8000,14:6000,16:4000,18:1500,20:500", help="n:systems,...")
    ap.add_argument("--data", default=None, help="dataset .npz (read if present, else generated and written)")
    ap.add_argument("--params", default=None, help="trained parameters .npy (read if present, else trained)")
    ap.add_argument("--eval", default="24:8", help="held-out n:count,...")
    ap.add_argument("--epochs", type=float, default=1.0, help="scale of the default training schedule")
    ap.add_argument("--out", default=None, help="JSON report")
    a = ap.parse_args(argv)

    def log(rec):
        print(json.dumps(rec), flush=True)

    report = {}
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
    X, Y = dataset(train_d)
    Xv, Yv = dataset(val_d)
    mlp = Mlp(seed=0)
    if a.params and os.path.exists(a.params):
        mlp.params = np.load(a.params)
    else:
        sched = [(max(1, int(round(e * a.epochs))), lr) for e, lr in ((60, 1e-3), (40, 3e-4), (30, 1e-4))]
        t0 = time.time()
        losses = train(mlp, X, Y, schedule=sched)
        report["train_seconds"] = round(time.time() - t0, 2)
        report["train_loss_first_last"] = [losses[0], losses[-1]]
        if a.params:
            np.save(a.params, mlp.params)
    report["train_samples"] = int(len(X))
    report["val_loss"] = mlp.loss_grad(Xv, Yv)[0]
    P = mlp.predict(Xv)
    report["val_max_density_err"] = float(np.abs(P[:, 0] - Yv[:, 0]).max())
    report["val_mean_density_err"] = float(np.abs(P[:, 0] - Yv[:, 0]).mean())
    log({k: report[k] for k in report if k != "generate"})
    rows = []
    for n, count in _pairs(a.eval):
        rows += evaluate(mlp, n, count, log=log)
    report["eval"] = rows
    for n in sorted({r["n"] for r in rows}):
        rs = [r for r in rows if r["n"] == n]
        tc, tw = sum(r["cold_seconds"] for r in rs), sum(r["warm_seconds"] for r in rs)
        report[f"summary_n{n}"] = {"systems": len(rs), "cold_seconds": round(tc, 3), "warm_seconds": round(tw, 3),
                                   "wall_time_ratio": round(tc / tw, 3),
                                   "median_speedup": float(np.median([r["speedup"] for r in rs])),
                                   "max_density_diff": max(r["max_density_diff"] for r in rs),
                                   "all_converged": all(r["cold_converged"] and r["warm_converged"] for r in rs)}
        log(report[f"summary_n{n}"])
    if a.out:
        with open(a.out, "w") as f:
            json.dump(report, f, indent=1)
    mlp.close()


if __name__ == "__main__":
    main()
