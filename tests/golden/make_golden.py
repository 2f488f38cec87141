#!/usr/bin/env python3
"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Run here, where the reference sources exist: `make -C oracle` first builds the
stock binary (oracle/_ref/masterEquation, reference sources compiled in place,
no GMP) and the reference-linked harness (oracle/_ref/libtasep_ref.so).

* stock/<case>/   output files of the stock binary (probabilities with %.20g,
                  densities, covariance, window observables) and run.json with
                  the command line and the lines it printed about the exit;
* harness/*.npz   final states of the reference's step code started from the
                  empty lattice (the binary can only start uniform), with the
                  exit bookkeeping;
* mpa.json        exact matrix-product steady-state densities (oracle/mpa.py).
"""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from oracle import mpa  # noqa: E402


def write_vec(path, v, fmt="%.17g"):
    with open(path, "w") as f:
        f.write(" ".join(fmt % x for x in v) + "\n")


def rates(n, seed):
    rng = np.random.default_rng(seed)
    r = np.empty(n + 1)
    r[0], r[n] = rng.uniform(0.1, 1.0, 2)
    r[1:n] = np.clip(rng.lognormal(0.0, 0.5, n - 1), 0.1, 5.0)
    return r


STOCK_CASES = {
    # config 1 as the reference is coded: uniform start, 1e-7*h rule, -f path
    "cfg1_f": {"args": ["-n", "10", "--alpha", "0.6", "--beta", "0.4", "--gamma", "1.0", "-t", "0", "-T", "300",
                        "-s", "30000", "-f"]},
    # inhomogeneous rates from a file, matrix-free per-row path
    "n7_rows": {"rates": (7, 11), "args": ["-n", "7", "-t", "0", "-T", "40", "-s", "4000"]},
    # inhomogeneous rates, -f path, all outputs
    "n8_f": {"rates": (8, 12), "args": ["-n", "8", "-t", "0", "-T", "60", "-s", "6000", "-f"]},
    # time-variant rates (per-row path, no exit test)
    "n5_timevar": {"rates": (5, 13), "timevar": True,
                   "args": ["-n", "5", "-t", "0", "-T", "6", "-s", "600", "--time-var"]},
    # snapshots every 50 steps (-a): timed files and per-snapshot matrix directories
    "n7_anim": {"rates": (7, 14), "args": ["-n", "7", "-t", "0", "-T", "3", "-s", "300", "-f", "-a", "50"]},
}


def run_stock(name, spec, outdir):
    tmp = tempfile.mkdtemp(prefix="golden_")
    try:
        args = list(spec["args"])
        files = {}
        if "rates" in spec:
            n, seed = spec["rates"]
            r = rates(n, seed)
            write_vec(os.path.join(tmp, "rates.txt"), r)
            args += ["-i", "rates.txt"]
            files["rates.txt"] = r.tolist()
            if spec.get("timevar"):
                rng = np.random.default_rng(seed + 100)
                tv = {"function-type": "".join("scl"[k] + " " for k in rng.integers(0, 3, n + 1)).split(),
                      "amplitude": (0.5 * r).tolist(), "period": rng.uniform(0.5, 2.0, n + 1).tolist(),
                      "offset": rng.uniform(0.0, 1.0, n + 1).tolist(), "constant": r.tolist()}
                with open(os.path.join(tmp, "ft.txt"), "w") as f:
                    f.write(" ".join(tv["function-type"]) + "\n")
                for k in ("amplitude", "period", "offset", "constant"):
                    write_vec(os.path.join(tmp, f"{k}.txt"), tv[k])
                args += ["--function-type", "ft.txt", "--amplitude", "amplitude.txt", "--period", "period.txt",
                         "--offset", "offset.txt", "--constant", "constant.txt"]
                files["timevar"] = tv
        args += ["-o", "out"]
        p = subprocess.run([O.REF_BIN] + args, cwd=tmp, capture_output=True, text=True, stdin=subprocess.DEVNULL)
        text = p.stdout.replace("\r", "\n")
        info = {"argv": args, "returncode": p.returncode, **files}
        for key, pat in (("convergence_after", r"Convergence after (\d+) steps"),
                         ("sim_time", r"Simulation time elapsed: ([0-9.]+)\n"),
                         ("checksum", r"Checksum over result vector: ([0-9.]+)")):
            m = re.findall(pat, text)
            info[key] = m[-1] if m else None
        dst = os.path.join(outdir, "stock", name)
        os.makedirs(dst, exist_ok=True)
        for fn in sorted(os.listdir(tmp)):
            if fn.startswith("out") and os.path.isfile(os.path.join(tmp, fn)):
                shutil.copy(os.path.join(tmp, fn), os.path.join(dst, fn))
            elif fn.startswith("out") and os.path.isdir(os.path.join(tmp, fn)):
                shutil.copytree(os.path.join(tmp, fn), os.path.join(dst, fn), dirs_exist_ok=True)
        with open(os.path.join(dst, "run.json"), "w") as f:
            json.dump(info, f, indent=1)
        print(name, "rc", p.returncode, "convergence", info["convergence_after"], sorted(os.listdir(dst)))
    finally:
        shutil.rmtree(tmp)


def run_harness(outdir):
    os.makedirs(os.path.join(outdir, "harness"), exist_ok=True)
    cases = {
        # config 1 as specified: empty start, 1e-10*h rule, 10000 steps (h = 0.01)
        "cfg1_empty": dict(n=10, r=np.array([0.6] + [1.0] * 9 + [0.4]), steps=10000, tol=1e-10),
        # same lattice run to convergence
        "cfg1_empty_converged": dict(n=10, r=np.array([0.6] + [1.0] * 9 + [0.4]), steps=200000, tol=1e-10),
        "n9_inhom": dict(n=9, r=rates(9, 21), steps=3000, tol=1e-10),
    }
    for name, c in cases.items():
        x, res = O.ref_run(c["n"], c["r"], h=0.01, steps=c["steps"], init=O.INIT_EMPTY, stop_tol=c["tol"],
                           use_csr=True)
        np.savez_compressed(os.path.join(outdir, "harness", name + ".npz"), x=x, rates=c["r"],
                            steps=c["steps"], tol=c["tol"], **{k: v for k, v in res.items()})
        print(name, res)


def run_mpa(outdir):
    out = []
    for n, a, b in [(6, 0.3, 0.5), (8, 0.9, 0.9), (8, 0.3, 0.7), (10, 0.6, 0.4), (12, 1.2, 0.35)]:
        rho = mpa.densities(n, a, b)
        out.append({"n": n, "alpha": a, "beta": b, "rho": [float(v) for v in rho],
                    "rho_exact": [f"{v.numerator}/{v.denominator}" for v in rho]})
    with open(os.path.join(outdir, "mpa.json"), "w") as f:
        json.dump(out, f, indent=1)


def main():
    if not os.path.exists(O.REF_BIN):
        sys.exit("build the reference first: make -C oracle")
    only = sys.argv[1:]  # optional: regenerate only these stock cases
    for name, spec in STOCK_CASES.items():
        if not only or name in only:
            run_stock(name, spec, HERE)
    if only:
        return
    run_harness(HERE)
    run_mpa(HERE)


if __name__ == "__main__":
    main()
