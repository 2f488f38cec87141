#!/usr/bin/env python3
"""Benchmark: classical-RK4 steps/s of the TASEP master equation at n=28 (FP64).

Workload (one step = one classical RK4 step = four generator applications on
2^28 states): n=28, site-inhomogeneous rates from seed 1 - alpha, beta ~
U[0.1, 1.0], 27 hop rates lognormal(0, 0.5) clipped to [0.1, 5] - h = 0.01,
empty-lattice start.  Data are synthetic (the rates are the workload).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours: one process per GPU (torchrun for N > 1), each integrating its own
replica (the path does not shard; no data-path collective).  Timing: CUDA
events on the library's stream around K steps, barrier + synchronize on both
sides, max over ranks.  Every vector (2 GiB) is larger than L2, so no flush
is needed between steps.  `e2e` repeats the measurement through the public
API with host buffers: the initial state is copied from pinned host memory,
K steps run, and the final probability vector is copied back, all inside the
timed region.

reference: the reference's own CPU step (src/lib/solv.c rk4_step x4 + the
serial update of src/masterEquation.c:639-642), compiled from the reference
sources into oracle/_ref, timed on the host cores with all threads over all
2^28 rows of the n=28 generator (CSR of about 52 GB, built untimed) when the
host has the memory, else on a bounded row sample scaled to all rows and
marked "extrapolated".  The line records the host's CPU model, core count and
memory.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK4 steps/s at n=28 (FP64 classical RK4, 4 generator applications per step)"
UNIT = "steps/s"

# algorithmic bytes per state of each kernel: the vectors it must read and write once
ALG_BYTES = {
    # constant-rate RK4 in factored form: v1 = z x, v2 = (z - r) v1, w = (z + p) v2,
    # x' = x + (z w + q v2) / 24 (each sweep reads its gathered vector once)
    ("meq_ref_step", 0): 16, ("meq_rk4_h1", 0): 16, ("meq_rk4_h2", 0): 16, ("meq_rk4_h3", 0): 16,
    ("meq_rk4_h4", 0): 32, ("meq_rk4_h1", 1): 12, ("meq_rk4_h2", 1): 8, ("meq_rk4_h3", 1): 8,
    ("meq_rk4_h4", 1): 24,
    # time-variant RK4: materialised stage inputs (u2, u3, u4), k recovered in the last stage
    ("meq_rk4_u1", 0): 16, ("meq_rk4_u2", 0): 24, ("meq_rk4_u3", 0): 24, ("meq_rk4_u4", 0): 40,
}
STEP_BYTES = {(1, 0): 80, (1, 1): 52, (0, 0): 16, (1, 0, "timevar"): 104}


def config_rates(n, seed=1):
    """alpha, beta ~ U[0.1,1]; n-1 hops lognormal(0,0.5) clipped to [0.1,5]."""
    rng = np.random.default_rng(seed)
    a, b = rng.uniform(0.1, 1.0, 2)
    hops = np.clip(rng.lognormal(0.0, 0.5, n - 1), 0.1, 5.0)
    return np.concatenate([[a], hops, [b]])


def config_timevar(n, seed=1):
    """The time-variant run on the same lattice: r_i(t) = r_i (1 + 0.5 sin(w_i t)),
    w_i ~ U[0.5, 2] drawn after the rates from the same stream, in the
    reference's function form A sin(w t + phi) + c (src/lib/matvec.c:44-68)."""
    rng = np.random.default_rng(seed)
    rng.uniform(0.1, 1.0, 2)
    rng.lognormal(0.0, 0.5, n - 1)
    w = rng.uniform(0.5, 2.0, n + 1)
    r = config_rates(n, seed)
    return {"type": np.zeros(n + 1, dtype=np.int32), "amplitude": 0.5 * r, "period": w,
            "offset": np.zeros(n + 1), "constant": r}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"tasep_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) == 6 and parts[0].isdigit():
                    rows.append(parts)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [int(r[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[2 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": int(rows[0][1]), "reasons": reasons,
                "samples": len(rows)}


def dist_setup(gpus, backend="nccl"):
    """One process per GPU (torchrun): the process group only carries the
    barrier and the max-over-ranks time; each rank integrates its own replica."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        return dist, rank, world, local
    return None, 0, 1, 0


def max_over_ranks(dist, x, device="cuda"):
    """The largest of every rank's x (every rank calls this at the same point)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(world, steps, ms):
    """Whole-job steps/s: every replica did `steps` steps in at most `ms`."""
    return world * steps / (ms / 1000.0)


def host_info():
    """CPU model, logical cores and memory of this host (for the CPU baseline)."""
    info = {"cpu_model": None, "logical_cpus": os.cpu_count(), "mem_total_gb": None, "mem_available_gb": None}
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    info["cpu_model"] = line.split(":", 1)[1].strip()
                    break
        with open("/proc/meminfo") as f:
            for line in f:
                k, v = line.split(":", 1)
                if k in ("MemTotal", "MemAvailable"):
                    info["mem_total_gb" if k == "MemTotal" else "mem_available_gb"] = round(
                        int(v.split()[0]) / 1048576.0, 1)
    except OSError:
        pass
    return info


def reference_full_bytes(n):
    """Host memory of the reference's -f step on all rows: CSR + 6 vectors."""
    dim = 1 << n
    nnz = 2 * dim + (dim >> 2) * (n - 1)
    return 8 * (dim + 1) + 16 * nnz + 6 * 8 * dim


def cpu_baseline_sample(n, rates, h, target_s=15.0):
    """Reference -f step on a row sample; returns (steps/s scaled to all rows, info)."""
    import oracle as O
    if not O.ref_available():
        return None
    threads = O.ref().refh_max_threads()
    rows = 1 << min(n, 22)
    secs, _ = O.ref_time_sample(n, rows, rates, h, reps=1, nthreads=threads)
    if secs <= 0:
        return None
    rows = min(1 << n, 1 << 25)
    est = secs * rows / float(1 << min(n, 22))
    reps = int(min(50, max(2, target_s / max(est, 1e-3))))
    secs, nnz = O.ref_time_sample(n, rows, rates, h, reps=reps, nthreads=threads)
    if secs <= 0:
        return None
    value = (rows / float(1 << n)) / secs
    return value, {"cores": threads, "sample": f"reference rk4_step x4 + serial update over rows "
                   f"[0, 2^{int(np.log2(rows))}) of the 2^{n}-state generator ({nnz} CSR entries), "
                   f"{reps} timed steps of {secs:.3f} s each, scaled to all rows (a bounded sample; "
                   f"bench.py --impl reference times all rows)", "host": host_info()}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle as O
    n = args.n
    rates = config_rates(n)
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"n={n} seed-1 inhomogeneous rates, h=0.01, empty start",
                       "n": n, "integrator": "reference rk4_step (four identical stage gathers)"}}
    if not O.ref_available():
        line["unavailable"] = "oracle/_ref was not built (reference sources absent when building)"
        print(json.dumps(line))
        return 0
    threads = O.ref().refh_max_threads()
    host = host_info()
    need = reference_full_bytes(n)
    avail = (host["mem_available_gb"] or 0.0) * 1073741824.0
    if avail >= 1.15 * need:
        # the whole generator: every one of the 2^n rows, as the reference runs it
        warm = min(args.warmup, 2)
        secs, build, nnz = O.ref_time_full(n, rates, 0.01, warm=warm, reps=args.steps, nthreads=threads)
        if secs > 0:
            value = 1.0 / secs
            cb = {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "extrapolated": False,
                  "sample": f"all 2^{n} rows ({nnz} CSR entries, {need / 1e9:.1f} GB), {args.steps} timed "
                            f"steps after {warm} untimed; CSR set-up {build:.1f} s (untimed)",
                  "host": host}
    else:
        secs = -1.0
    if secs <= 0:
        rows = 1 << min(n, 22)
        s1, _ = O.ref_time_sample(n, rows, rates, 0.01, reps=1, nthreads=threads)
        per_step_budget = 60.0 / max(args.steps + 1, 1)
        rows = min(1 << n, 1 << 25, max(1 << 20, int(rows * per_step_budget / max(s1, 1e-3))))
        rows = 1 << int(np.log2(rows))
        secs, nnz = O.ref_time_sample(n, rows, rates, 0.01, reps=args.steps, nthreads=threads)
        value = (rows / float(1 << n)) / secs
        cb = {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "extrapolated": True,
              "sample": f"rows [0, 2^{int(np.log2(rows))}) of 2^{n} ({nnz} CSR entries), {args.steps} timed "
                        f"steps after 1 untimed, scaled to all rows: the whole generator needs "
                        f"{need / 1e9:.1f} GB of host memory, {host['mem_available_gb']} GB available",
              "host": host}
    line.update({"value": value, "ms_per_step": 1000.0 / value, "cpu_baseline": cb,
                 "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch
    import tasep_b200 as T
    dist, rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    n = args.n
    integ = {"rk4": T.INTEGRATOR_RK4, "ref": T.INTEGRATOR_REF}[args.integrator]
    prec = {"fp64": T.PRECISION_FP64, "mixed": T.PRECISION_MIXED}[args.precision]
    rates = config_rates(n)
    h = 0.01
    N = 1 << n
    m = T.Meq(n, integ, prec, device=local)
    m.set_rates(rates)
    tv = config_timevar(n) if args.timevar else None
    if tv is not None:
        m.set_timevar(tv["type"], tv["amplitude"], tv["period"], tv["offset"], tv["constant"])
    m.init(T.INIT_EMPTY)
    policy = m.cache_policy()
    stream = torch.cuda.ExternalStream(m.stream)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up
    m.enqueue_steps(h, args.warmup)
    m.synchronize()
    barrier()
    # timed: device-resident state
    m.profile(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        ev0.record(stream)
        m.enqueue_steps(h, args.steps, t0=args.warmup * h)
        ev1.record(stream)
        ev1.synchronize()
        barrier()
    ms = ev0.elapsed_time(ev1)
    prof = m.profile_read()
    m.profile(False)
    clocks = clk.summary()
    ms = max_over_ranks(dist, ms)
    value = replicas_value(world, args.steps, ms)

    # e2e through the public API with host buffers
    x_host = torch.zeros(N, dtype=torch.float64, pin_memory=True).numpy()
    x_host[0] = 1.0
    out_host = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.load(x_host)
    m.set_rates(rates)
    m.enqueue_steps(h, args.steps)
    m.store(out_host)
    e1.record(stream)
    e1.synchronize()
    barrier()
    ems = max_over_ranks(dist, e0.elapsed_time(e1))
    e2e_value = replicas_value(world, args.steps, ems)
    mass = float(out_host.sum())

    # roofline of the dominant kernel
    peak, peak_kind = peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][0]) if prof else None
    roof = None
    if dom:
        name, (tot_ms, cnt) = dom
        avg = tot_ms / cnt
        b = ALG_BYTES.get((name, prec), 0) * N
        achieved = b / (avg / 1000.0) / 1e9
        # DRAM traffic is not measured in this run (that needs ncu): it comes from
        # the stored capture of the same kernel, workload size and cache policy
        traffic, traffic_src = None, None
        tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
        if os.path.exists(tp):
            with open(tp) as f:
                tr = json.load(f)
            k = f"{name}/{args.precision}"
            rec = tr.get(k, {})
            if rec.get("n") == n and rec.get("l2_policy") == list(policy):
                traffic = rec["bytes_per_state"] * N
                traffic_src = f"stored ncu capture ({rec.get('source', 'profiles/ncu_traffic.json')}), not this run"
        kernel_ms = {k: v[0] / v[1] for k, v in prof.items()}
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                "traffic_source": traffic_src, "alg_bytes_per_launch": b, "avg_launch_ms": avg,
                "kernel_ms": kernel_ms,
                "kernel_frac": {k: ALG_BYTES.get((k, prec), 0) * N / (v / 1000.0) / 1e9 / peak
                                for k, v in kernel_ms.items()}}
    launches = int(sum(v[1] for v in prof.values()))
    step_alg = STEP_BYTES.get((integ, prec, "timevar") if args.timevar else (integ, prec), 0) * N
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_sample(n, rates, h)
        if cb is not None:
            cpu = {"value": cb[0], "unit": UNIT, "cores": cb[1]["cores"], "kind": "reference",
                   "extrapolated": True, "sample": cb[1]["sample"], "host": cb[1]["host"]}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == 0 else "f64 state / f32 stages", "data": "synthetic",
        "config": {"workload": f"n={n}: 2^{n} states, seed-1 inhomogeneous rates, h=0.01, empty start; "
                               f"{'classical RK4' if integ else 'reference step'}",
                   "n": n, "integrator": args.integrator, "precision": args.precision,
                   "rates": "time-variant r_i(t) = r_i (1 + 0.5 sin(w_i t)), w_i ~ U[0.5, 2], seed 1"
                            if args.timevar else "constant",
                   "replicas": world, "l2": "inputs larger than L2 (8*2^n bytes per vector)",
                   "l2_policy": {"near_bits": policy[0], "flags": policy[1]},
                   "hbm_step_bytes_algorithmic": step_alg,
                   "step_hbm_gbs_algorithmic": step_alg / (ms / args.steps / 1000.0) / 1e9},
        "roofline": roof, "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": (8 * N + 8 * (n + 1)) / args.steps,
                "d2h_bytes_per_step": 8 * N / args.steps, "mass_after": mass},
        "gpu_launches": launches, "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line))
    m.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=28, help="lattice length (the benchmark is n=28)")
    ap.add_argument("--integrator", choices=["rk4", "ref"], default="rk4")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--timevar", action="store_true",
                    help="the time-variant run of the same lattice (RK4, FP64; rates evaluated per stage)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        ap.error("--warmup must be at least 3")
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
