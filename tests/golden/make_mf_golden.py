#!/usr/bin/env python3
"""Regenerates tests/golden/mf_full/ from the reference's mean-field program.

Run here, where the reference sources exist: `make -C oracle ref` builds the
stock program oracle/_ref/mf_full (src/mf_full.c compiled in place).  Each
case runs it with the closure order -c, the rates (-a/-b/-g or an -i file),
-t/-T/-s and the RK4 solver (-m r), and keeps the densities it writes to -o
(one line "site, density" per site, printed with %lf by save_state_singles,
src/mf_full.c:1737-1746).  cases.json holds the arguments and the parsed
densities; tests/test_closure.py holds tasep_b200/closure.py to them.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "mf_full")
MF = os.path.join(ROOT, "oracle", "_ref", "mf_full")


def rates(n, seed):
    rng = np.random.default_rng(seed)
    r = np.empty(n + 1)
    r[0], r[n] = rng.uniform(0.1, 1.0, 2)
    r[1:n] = np.clip(rng.lognormal(0.0, 0.5, n - 1), 0.1, 5.0)
    return r


CASES = []
for order in (1, 2, 3, 4):  # homogeneous hops, not yet stationary at T = 10
    CASES.append({"name": f"n8_hom_c{order}", "n": 8, "order": order, "t": 0.0, "T": 10.0, "s": 1000,
                  "rates": [0.3] + [1.0] * 7 + [0.5]})
for order in (2, 3):  # inhomogeneous rates from a file
    CASES.append({"name": f"n10_inhom_c{order}", "n": 10, "order": order, "t": 0.0, "T": 20.0, "s": 2000,
                  "rates": rates(10, 21).tolist()})
# close to the closed hierarchy's steady state
CASES.append({"name": "n9_steady_c3", "n": 9, "order": 3, "t": 0.0, "T": 200.0, "s": 10000,
              "rates": rates(9, 22).tolist()})
# one below the lattice length: only the full-lattice window is closed
CASES.append({"name": "n6_c5", "n": 6, "order": 5, "t": 0.0, "T": 5.0, "s": 500,
              "rates": rates(6, 23).tolist()})


def run_case(case, tmp):
    n = case["n"]
    r = case["rates"]
    args = [MF, "-n", str(n), "-c", str(case["order"]), "-t", repr(case["t"]), "-T", repr(case["T"]),
            "-s", str(case["s"]), "-m", "r"]
    homogeneous = all(x == r[1] for x in r[1:n])
    if homogeneous:
        args += ["-a", repr(r[0]), "-b", repr(r[n]), "-g", repr(r[1])]
    else:
        rf = os.path.join(tmp, "rates.txt")
        with open(rf, "w") as f:
            f.write(" ".join("%.17g" % x for x in r) + "\n")
        args += ["-i", rf]
    out = os.path.join(tmp, "out.txt")
    args += ["-o", out]
    subprocess.run(args, cwd=tmp, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    rho = []
    with open(out) as f:
        for line in f:
            if "," in line:
                s, v = line.split(",")
                assert int(s) == len(rho)
                rho.append(float(v))
    assert len(rho) == n
    shown = [a if not a.startswith(tmp) else os.path.basename(a) for a in args[1:]]
    return {**case, "args": shown, "rho": rho}


def main():
    if not os.path.exists(MF):
        sys.exit("oracle/_ref/mf_full missing: run make -C oracle ref first")
    os.makedirs(OUT, exist_ok=True)
    res = []
    with tempfile.TemporaryDirectory() as tmp:
        for c in CASES:
            res.append(run_case(c, tmp))
    with open(os.path.join(OUT, "cases.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(f"wrote {len(res)} cases to {OUT}")


if __name__ == "__main__":
    main()
