"""Batched parameter sweep of the master equation (tasep_batch_* in libtasep_cuda.so).

The reference runs bin/masterEquation once per rate vector; a sweep here is
one batch on one GPU.  The standard sweep is 1024 systems at n = 16: entry
and exit rates (alpha, beta) on a 32 x 32 grid over [0.05, 1.5]^2 (system
s = 32 * a + b for grid indices a of alpha and b of beta) and 15 hop rates per
system ~ U[0.5, 1.5] from numpy's default_rng(2); h = 0.01, empty lattice,
each system classical RK4 to its own exit rule (|dP| < 1e-10 h on more than
100 consecutive steps, src/masterEquation.c:670-679).

    python -m tasep_b200.sweep [--precision fp64|mixed|both] [--schedule S] [--out report.json]
    python -m tasep_b200.sweep --cost-profile [--schedule S]

writes per-system exit steps and final densities, the sweep's wall time and
the schedule the autotuner chose; --cost-profile prints the time of one step
against the number of systems running.
"""
from __future__ import annotations

import json
import time

import numpy as np

from . import Batch, INIT_EMPTY, PRECISION_FP64, PRECISION_MIXED

GRID = 32
N_SWEEP = 16


def sweep_rates(n=N_SWEEP, grid=GRID, lo=0.05, hi=1.5, seed=2):
    """(grid*grid, n+1) rates: alpha, beta on the grid, hops ~ U[0.5, 1.5]."""
    ab = np.linspace(lo, hi, grid)
    hops = np.random.default_rng(seed).uniform(0.5, 1.5, (grid * grid, n - 1))
    a = np.repeat(ab, grid)
    b = np.tile(ab, grid)
    return np.column_stack([a, hops, b])


def run_sweep(rates, precision=PRECISION_FP64, h=0.01, max_steps=2_000_000, stop_tol=1e-10, schedule=-1,
              device=-1):
    """Runs every system of `rates` to its exit rule in one batch; returns
    (per-system results, densities (nsys, n) in site order, seconds, schedule used)."""
    R = np.asarray(rates, dtype=np.float64)
    nsys, n = R.shape[0], R.shape[1] - 1
    with Batch(n, nsys, precision, device=device) as b:
        b.set_rates(R)
        b.init(INIT_EMPTY)
        t0 = time.perf_counter()
        res, used = b.run(h, max_steps, stop_tol=stop_tol, schedule=schedule)
        sec = time.perf_counter() - t0
        rho = b.densities()[:, ::-1]
    return res, rho, sec, used


def cost_profile(n=N_SWEEP, counts=(1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024), steps=512, schedule=-1,
                 precision=PRECISION_FP64):
    """Device time per step of the batched integrator against the number of
    systems running (the standard sweep's first systems, no exit rule): the
    cost a sweep pays at each point of its retirement curve."""
    R = sweep_rates(n)
    out = []
    for k in counts:
        with Batch(n, k, precision) as b:
            b.set_rates(R[:k])
            b.init(INIT_EMPTY)
            b.run(0.01, 32, exit_rule=False, schedule=schedule)  # warm-up (and the autotuner's probes)
            t0 = time.perf_counter()
            b.run(0.01, steps, exit_rule=False, schedule=schedule)
            sec = time.perf_counter() - t0
            sched, spc, ctas = b.last_config()
        out.append({"systems": k, "us_per_step": sec / steps * 1e6, "schedule": sched, "states_per_cta": spc,
                    "ctas_per_system": ctas})
    return out


def report(res, rho, sec, used, precision):
    steps = np.array([r["steps_done"] for r in res], dtype=np.int64)
    n = rho.shape[1]
    applications = 4 * int(steps.sum()) * (1 << n)  # generator row applications
    return {"precision": "fp64" if precision == PRECISION_FP64 else "mixed", "systems": len(res),
            "converged": int(sum(r["converged"] for r in res)), "seconds": round(sec, 3),
            "schedule": used, "steps_min": int(steps.min()), "steps_median": int(np.median(steps)),
            "steps_max": int(steps.max()), "steps_total": int(steps.sum()),
            "state_applications_per_s": applications / sec,
            "steps": steps.tolist(), "rho": np.round(rho, 12).tolist()}


def main(argv=None):
    import argparse

    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="both")
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--n", type=int, default=N_SWEEP)
    ap.add_argument("--schedule", type=int, default=-1,
                    help="-1 automatic (tile engines), 0/1 a tile engine, 2 cluster-resident")
    ap.add_argument("--cost-profile", action="store_true",
                    help="only time one step against the number of running systems")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    if a.cost_profile:
        for rec in cost_profile(a.n, schedule=a.schedule):
            print(json.dumps(rec), flush=True)
        return
    R = sweep_rates(a.n, a.grid)
    out = {"workload": f"{a.grid * a.grid} systems, n={a.n}, (alpha, beta) on a {a.grid}x{a.grid} grid over "
                       f"[0.05, 1.5]^2, hops U[0.5, 1.5] seed 2, h=0.01, empty start, exit 1e-10*h / 100 steps",
           "runs": []}
    precs = {"fp64": [PRECISION_FP64], "mixed": [PRECISION_MIXED], "both": [PRECISION_FP64, PRECISION_MIXED]}
    for p in precs[a.precision]:
        rec = report(*run_sweep(R, p, schedule=a.schedule), p)
        out["runs"].append(rec)
        print(json.dumps({k: v for k, v in rec.items() if k not in ("steps", "rho")}), flush=True)
    if len(out["runs"]) == 2:
        d = np.abs(np.array(out["runs"][0]["rho"]) - np.array(out["runs"][1]["rho"]))
        out["mixed_vs_fp64_max_density_diff"] = float(d.max())
        print(json.dumps({"mixed_vs_fp64_max_density_diff": float(d.max())}), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f)


if __name__ == "__main__":
    main()
