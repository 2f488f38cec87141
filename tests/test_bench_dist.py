"""bench.py's multi-GPU plumbing on CPU: two gloo ranks (replicas only, no
data-path collective), the max-over-ranks time and the whole-job value, and
the reference arm's rank rule under torchrun."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist, r, w, local = bench.dist_setup(world, backend="gloo")
    assert (r, w, local) == (rank, world, rank)
    ms = 100.0 + 50.0 * rank  # this rank's timed region
    worst = bench.max_over_ranks(dist, ms, device="cpu")
    dist.barrier()
    out[rank] = (worst, bench.replicas_value(w, 40, worst))
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    # both ranks see the slowest rank's 150 ms; 2 replicas x 40 steps in 0.15 s
    assert res[0] == res[1] == (150.0, 2 * 40 / 0.150)


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    os.environ.pop("WORLD_SIZE", None)
    assert bench.dist_setup(1)[0] is None
    assert bench.max_over_ranks(None, 12.5) == 12.5


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == ""
