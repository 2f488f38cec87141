"""Memory-limit runs: mixed precision at n = 30, 32, 33 (homogeneous hop rate 1).

    python -m tasep_b200.memlimit [--steps30 S] [--steps33 K] [--out report.json]

* n = 30, low density (alpha=0.3, beta=0.7) and maximal current
  (alpha=beta=0.9): the FP64 and the mixed integrator (FP64 state, FP32 stage
  vectors) from the empty lattice for S steps; densities of both, their
  largest difference, steps/s of both.
* n = 32 and 33 in the mixed layout (20 B per state: 85.9 GB and 171.8 GB):
  low density started from its exact stationary measure (the Bernoulli(0.3)
  product measure, stationary on alpha + beta = 1) and maximal current from
  the empty lattice, K steps each: steps/s, the L1 norm of the last increment,
  densities and total probability.
"""
from __future__ import annotations

import json
import time

import numpy as np

from . import INIT_EMPTY, INTEGRATOR_RK4, Meq, PRECISION_FP64, PRECISION_MIXED, footprint, init_pair_markov

PHASES = {"low_density": (0.3, 0.7), "maximal_current": (0.9, 0.9)}


def homogeneous(n, a, b):
    return np.array([a] + [1.0] * (n - 1) + [b])


def timed_run(m, steps, h=0.01):
    m.synchronize()
    t0 = time.perf_counter()
    res = m.run(h, steps, exit_rule=False)
    sec = time.perf_counter() - t0
    obs = m.observables()
    return res, obs, sec


def n30(steps, log=print):
    out = {}
    for name, (a, b) in PHASES.items():
        rec = {"alpha": a, "beta": b, "steps": steps}
        for prec, tag in ((PRECISION_FP64, "fp64"), (PRECISION_MIXED, "mixed")):
            with Meq(30, INTEGRATOR_RK4, prec) as m:
                m.set_rates(homogeneous(30, a, b))
                m.init(INIT_EMPTY)
                res, obs, sec = timed_run(m, steps)
            rec[tag] = {"steps_per_s": steps / sec, "last_checksum": res["last_checksum"],
                        "mass": obs["mass"], "rho_sites": obs["rho"][::-1].tolist()}
        rec["max_density_diff"] = float(np.max(np.abs(np.array(rec["fp64"]["rho_sites"]) -
                                                      np.array(rec["mixed"]["rho_sites"]))))
        out[name] = rec
        log(json.dumps({"n": 30, "phase": name, "max_density_diff": rec["max_density_diff"],
                        "fp64_steps_per_s": rec["fp64"]["steps_per_s"],
                        "mixed_steps_per_s": rec["mixed"]["steps_per_s"]}))
    return out


def large(n, steps, log=print):
    out = {"n": n, "bytes": footprint(n, INTEGRATOR_RK4, PRECISION_MIXED)}
    for name, (a, b) in PHASES.items():
        with Meq(n, INTEGRATOR_RK4, PRECISION_MIXED) as m:
            m.set_rates(homogeneous(n, a, b))
            if name == "low_density":
                init_pair_markov(m, np.full(n, a), np.zeros(n - 1))  # exact stationary measure
                start = "Bernoulli(0.3) product measure (stationary)"
            else:
                m.init(INIT_EMPTY)
                start = "empty lattice"
            res, obs, sec = timed_run(m, steps)
        rec = {"alpha": a, "beta": b, "start": start, "steps": steps, "steps_per_s": steps / sec,
               "last_checksum": res["last_checksum"], "mass": obs["mass"], "rho_sites": obs["rho"][::-1].tolist()}
        out[name] = rec
        log(json.dumps({"n": n, "phase": name, **{k: v for k, v in rec.items() if k != "rho_sites"}}))
    return out


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--steps30", type=int, default=2000)
    ap.add_argument("--steps33", type=int, default=20)
    ap.add_argument("--sizes", default="32,33")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    rep = {"n30": n30(a.steps30)}
    for n in [int(v) for v in a.sizes.split(",") if v]:
        rep[f"n{n}"] = large(n, a.steps33)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
