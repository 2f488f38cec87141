"""The drop-in masterEquation program.

CPU tests: option handling and error paths (exit code -1 = 255 and the
reference's messages, src/masterEquation.c:239-429), which need no device.
GPU tests: the program run with the stock reference binary's own command
lines (tests/golden/stock/*/run.json) writes the same files - the probability
file byte for byte - as the reference did.
"""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
import tasep_b200 as T

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "stock")
CLI = T.CLI_PATH


def run(args, cwd, stdin=""):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, input=stdin, timeout=600)


def test_cli_built():
    assert os.access(CLI, os.X_OK)


def test_unknown_option_prints_usage_and_fails(tmp_path):
    p = run(["--bogus"], tmp_path)
    assert p.returncode == 255 and "Usage:" in p.stdout


def test_f_with_time_var_is_rejected(tmp_path):
    p = run(["-f", "--time-var", "-n", "4"], tmp_path)
    assert p.returncode == 255
    assert "ERROR: -f cannot be selected in combination with --time-var" in p.stderr


def test_missing_alpha_is_rejected(tmp_path):
    p = run(["-n", "5", "--beta", "0.5", "-t", "0", "-T", "1", "-s", "10"], tmp_path)
    assert p.returncode == 255 and "No value for alpha found" in p.stderr


def test_missing_values_are_prompted(tmp_path):
    # n, the n+1 rates, T, t, steps from standard input, as the reference asks for them
    p = run(["-o", "o"], tmp_path, stdin="4\n0.5 1 1 1 0.5\n1\n0\n10\n")
    assert "Enter length: " in p.stdout
    assert "Enter 5 probabilities: " in p.stdout
    assert "No end time found. Please enter: " in p.stdout
    assert "No start time found. Please enter: " in p.stdout
    assert "No step number found. Please Enter: " in p.stdout


def test_bad_rate_file_is_reported(tmp_path):
    (tmp_path / "r.txt").write_text("0.5 1\n")
    p = run(["-n", "4", "-i", "r.txt", "-t", "0", "-T", "1", "-s", "10", "-o", "o"], tmp_path)
    assert p.returncode == 255 and "Issue while reading from jump rate file name" in p.stderr


# ---------------------------------------------------------------- GPU ---------

CASES = ["cfg1_f", "n7_rows", "n8_f", "n5_timevar", "n7_anim"]


def _prepare(name, tmp_path):
    d = os.path.join(GOLD, name)
    with open(os.path.join(d, "run.json")) as f:
        info = json.load(f)
    if "rates.txt" in info:
        (tmp_path / "rates.txt").write_text(" ".join("%.17g" % v for v in info["rates.txt"]) + "\n")
    if "timevar" in info:
        tv = info["timevar"]
        (tmp_path / "ft.txt").write_text(" ".join(tv["function-type"]) + "\n")
        for k in ("amplitude", "period", "offset", "constant"):
            (tmp_path / f"{k}.txt").write_text(" ".join("%.17g" % v for v in tv[k]) + "\n")
    return d, info


def _floats(path):
    return np.array([float(t) for t in open(path).read().replace(",", " ").replace(":", " ").split()
                     if t.replace(".", "", 1).replace("-", "", 1).replace("e", "", 1).isdigit()])


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_drop_in_matches_stock_binary_files(name, tmp_path):
    d, info = _prepare(name, tmp_path)
    # the reference binary's coded exit tolerance is 1e-7 (src/masterEquation.c:186)
    p = run(info["argv"] + ["--stop-tol", "1e-7"], tmp_path)
    assert p.returncode == 0, p.stderr
    if info["convergence_after"] is not None:
        assert f"Convergence after {info['convergence_after']} steps" in p.stdout
    assert f"Simulation time elapsed: {info['sim_time']}" in p.stdout
    ours = sorted(f for f in os.listdir(tmp_path) if f.startswith("out"))
    theirs = sorted(f for f in os.listdir(d) if f.startswith("out"))
    assert ours == theirs
    # probabilities: byte-identical file.  Time-variant rates are evaluated on the
    # device with CUDA's sin/cos, which may differ from glibc's by an ulp, so that
    # case is held to the 1e-12 probability bar instead.
    mine, gold = open(os.path.join(tmp_path, "out"), "rb").read(), open(os.path.join(d, "out"), "rb").read()
    if "timevar" in info:
        pa = np.array([float(line.split()[1]) for line in mine.decode().splitlines()])
        pb = np.array([float(line.split()[1]) for line in gold.decode().splitlines()])
        assert np.max(np.abs(pa - pb)) <= 1e-12
    else:
        assert mine == gold
    # heat maps: byte-identical
    for fn in ("out_cov.ppm", "out_mulExpVa"):
        assert open(os.path.join(tmp_path, fn), "rb").read() == open(os.path.join(d, fn), "rb").read(), fn
    # printed observables: equal to the printed precision (values differ by rounding only)
    for fn in ("out_exp_values_fin.vec", "out_exp_values_fin.dat", "out_cov.mat", "out_closures",
               "out_error_guess", "out_high_order_point_fun"):
        a, b = _floats(os.path.join(tmp_path, fn)), _floats(os.path.join(d, fn))
        assert a.shape == b.shape and np.max(np.abs(a - b)) <= 1.5e-6, fn
    # the correlation file holds the correlation coefficient (the reference returns nothing there)
    n = int(info["argv"][info["argv"].index("-n") + 1])
    rows = [line.split() for line in open(os.path.join(tmp_path, "out_highcorr"))]
    assert [int(v) for v in rows[0]] == list(range(1, n - 2))
    assert len(rows) == 5 and all(len(r) == n - 2 for r in rows[1:])


@pytest.mark.gpu
def test_drop_in_snapshots_match_stock_binary(tmp_path):
    """-a 50: the timed density and probability files, and the per-snapshot
    covariance and product matrices with their pictures, as the stock binary
    wrote them (src/masterEquation.c:646-666, :1047-1110, :1197-1279,
    :1345-1417, :1516-1536)."""
    d, info = _prepare("n7_anim", tmp_path)
    p = run(info["argv"] + ["--stop-tol", "1e-7"], tmp_path)
    assert p.returncode == 0, p.stderr
    assert "Allocatng memory for animation data" in p.stdout
    for sub in ("out_covariance_data", "out_multExpval_data"):
        names = sorted(os.listdir(os.path.join(d, sub)))
        assert sorted(os.listdir(tmp_path / sub)) == names
        for fn in names:
            a, b = (tmp_path / sub / fn).read_bytes(), open(os.path.join(d, sub, fn), "rb").read()
            if fn.endswith(".ppm"):
                assert a.split(b"\n", 3)[:3] == b.split(b"\n", 3)[:3] and len(a) == len(b)
                assert max(abs(x - y) for x, y in zip(a, b)) <= 1, (sub, fn)
            else:
                fa, fb = _floats(tmp_path / sub / fn), _floats(os.path.join(d, sub, fn))
                assert fa.shape == fb.shape and np.max(np.abs(fa - fb)) <= 1.5e-6, (sub, fn)
    for fn in ("out_exp_timed.txt", "out_prb.txt"):
        fa, fb = _floats(tmp_path / fn), _floats(os.path.join(d, fn))
        assert fa.size > 0 and fa.shape == fb.shape and np.max(np.abs(fa - fb)) <= 1.5e-6, fn
    # timed 4-site correlations: same snapshot times and row lengths; the values
    # are the correlation coefficient (the reference function returns nothing)
    ours = [line.split() for line in open(tmp_path / "out_highcorr_timed")]
    gold = [line.split() for line in open(os.path.join(d, "out_highcorr_timed"))]
    assert [r[0] for r in ours] == [r[0] for r in gold]
    assert all(len(r) == 1 + 7 - 5 for r in ours)


@pytest.mark.gpu
def test_drop_in_rk4_empty_start_runs_to_the_exit_rule(tmp_path):
    """Config 1 as specified: empty lattice, 1e-10*h exit rule, classical RK4."""
    p = run(["-n", "10", "--alpha", "0.6", "--beta", "0.4", "--gamma", "1.0", "-t", "0", "-T", "2000", "-s",
             "200000", "--integrator", "rk4", "--init", "empty", "-o", "o", "--save-select", "ep"], tmp_path)
    assert p.returncode == 0, p.stderr
    assert "Convergence after" in p.stdout
    x = np.zeros(1 << 10)
    for line in open(tmp_path / "o"):
        b, v = line.split()
        x[int(b, 2)] = float(v)
    xo, ro = O.run(10, [0.6] + [1.0] * 9 + [0.4], h=0.01, steps=200000, integrator=O.INT_RK4, init=O.INIT_EMPTY)
    assert f"Convergence after {ro['steps_at_stop']} steps" in p.stdout
    assert np.max(np.abs(x - xo)) <= 1e-12
    # on alpha + beta = 1 the steady state is a product measure with density alpha
    vec = [float(v) for v in open(tmp_path / "o_exp_values_fin.vec").read().split(",")]
    assert max(abs(v - 0.6) for v in vec) < 1e-6


@pytest.mark.gpu
def test_drop_in_learned_warm_start(tmp_path):
    """--init learned starts from the pair-Markov measure of the shipped
    network's prediction (one step of h = 1e-30 leaves it as it was), the same
    measure the Python driver builds, and runs to the cold start's steady state."""
    from tasep_b200 import warmstart as ws
    n = 12
    r = ws.sample_rates(n, 1, np.random.default_rng(9))[0]
    (tmp_path / "rates.txt").write_text(" ".join("%.17g" % v for v in r) + "\n")
    p = run(["-n", str(n), "-i", "rates.txt", "-t", "0", "-T", "1e-30", "-s", "1", "--init", "learned",
             "--save-select", "p", "-o", "w"], tmp_path)
    assert p.returncode == 0, p.stderr
    assert "Initial vector from the learned warm start" in p.stdout
    x = np.zeros(1 << n)
    for line in open(tmp_path / "w"):
        b, v = line.split()
        x[int(b, 2)] = float(v)
    net = ws.pretrained()
    rho, cov = ws.predict_profile(net, r)
    net.close()
    with T.Meq(n, T.INTEGRATOR_RK4) as m:
        T.init_pair_markov(m, rho, cov)
        ref = m.store()
    assert np.max(np.abs(x - ref)) <= 1e-15
    common = ["-n", str(n), "-i", "rates.txt", "-t", "0", "-T", "3000", "-s", "300000", "--integrator", "rk4",
              "--save-select", "e"]
    assert run(common + ["--init", "learned", "-o", "a"], tmp_path).returncode == 0
    assert run(common + ["--init", "empty", "-o", "b"], tmp_path).returncode == 0
    va = [float(v) for v in open(tmp_path / "a_exp_values_fin.vec").read().split(",")]
    vb = [float(v) for v in open(tmp_path / "b_exp_values_fin.vec").read().split(",")]
    assert max(abs(u - v) for u, v in zip(va, vb)) <= 2e-6  # printed with %lf


@pytest.mark.gpu
def test_drop_in_resume_from_probability_file(tmp_path):
    args = ["-n", "9", "--alpha", "0.3", "--beta", "0.8", "-t", "0", "-T", "5", "-s", "500", "--save-select", "p"]
    assert run(args + ["-o", "a"], tmp_path).returncode == 0
    assert run(args + ["-o", "b", "--init-file", "a"], tmp_path).returncode == 0
    full = ["-n", "9", "--alpha", "0.3", "--beta", "0.8", "-t", "0", "-T", "10", "-s", "1000", "--save-select", "p"]
    assert run(full + ["-o", "c"], tmp_path).returncode == 0
    assert open(tmp_path / "b").read() == open(tmp_path / "c").read()
