"""Host side of the drop-in program without a GPU, compiled here into small
shared libraries: the window observables and the snapshot writers of
tasep_b200/host/me_output.c against the oracle's restatement of the
reference functions (src/masterEquation.c:32-143, :1047-1110, :1516-1536),
and the warm-start inputs of tasep_b200/host/me_warm.c against the Python
driver."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "tasep_b200", "host")
MAXN = 33


class Obs(C.Structure):
    _fields_ = [("n", C.c_int), ("y", C.c_double * MAXN), ("cov", C.c_double * (MAXN * MAXN)),
                ("mul", C.c_double * (MAXN * MAXN)), ("p4", C.c_double * ((MAXN - 3) * 16))]


class Snaps(C.Structure):
    _fields_ = [("n", C.c_int), ("dim", C.c_uint64), ("keep_probs", C.c_int), ("count", C.c_size_t),
                ("cap", C.c_size_t), ("obs", C.POINTER(Obs)), ("probs", C.POINTER(C.c_double)),
                ("corr", C.POINTER(C.c_double)), ("buf", C.POINTER(C.c_double))]


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    out = tmp_path_factory.mktemp("host") / "libmeout.so"
    subprocess.run(["gcc", "-std=c99", "-O2", "-shared", "-fPIC", "-D_DEFAULT_SOURCE", "-pthread", "-I", HOST,
                    "-I", os.path.join(ROOT, "include"), os.path.join(HOST, "me_output.c"), "-lm", "-o", str(out)],
                   check=True)
    L = C.CDLL(str(out))
    dp = C.POINTER(C.c_double)
    L.me_state_corr.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.me_state_corr.restype = C.c_double
    for f in ("me_win_corr", "me_win_error_guess", "me_win_closure"):
        getattr(L, f).argtypes = [C.POINTER(Obs), C.c_int, C.c_int]
        getattr(L, f).restype = C.c_double
    L.me_win_point.argtypes = [C.POINTER(Obs), C.c_int, C.c_int, C.c_int]
    L.me_win_point.restype = C.c_double
    L.me_write_prb_txt.argtypes = [C.c_char_p, C.POINTER(Snaps), C.c_double]
    L.me_write_exp_timed.argtypes = [C.c_char_p, C.POINTER(Snaps), C.c_double]
    L.me_write_highcorr_timed.argtypes = [C.c_char_p, C.POINTER(Snaps), C.c_double]
    return L


def _state(n, seed):
    x = np.random.default_rng(seed).random(1 << n) + 0.05
    return x / x.sum()


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_state_correlation_matches_oracle(host):
    n = 9
    x = _state(n, 1)
    for key, size in ((15, 4), (3, 2), (0, 2), (6, 3)):
        for off in range(1, n - size):
            a = host.me_state_corr(_dp(x), n, key, size, off)
            b = O.high_order_corr(x, key, size, off)
            assert a == pytest.approx(b, rel=1e-12, abs=1e-15)


def test_window_observables_from_marginals_match_oracle(host):
    n = 10
    x = _state(n, 2)
    ob = Obs()
    ob.n = n
    p4 = O.window4(n, x).ravel()
    for i, v in enumerate(p4):
        ob.p4[i] = v
    for off in range(1, n - 2):
        for key in range(4):
            assert host.me_win_corr(C.byref(ob), key, off) == pytest.approx(O.high_order_corr(x, key, 2, off),
                                                                             rel=1e-10)
        assert host.me_win_error_guess(C.byref(ob), 3, off) == pytest.approx(O.error_guess(x, 3, 2, off), rel=1e-10)
        assert host.me_win_closure(C.byref(ob), 3, off) == pytest.approx(O.pf_approx(x, 3, 2, off), rel=1e-10)
    for off in range(0, n - 3):
        assert host.me_win_point(C.byref(ob), 15, 4, off) == pytest.approx(O.point_func(x, 15, 4, off), rel=1e-12)


def test_snapshot_files_format(host, tmp_path):
    n, count = 6, 3
    dim = 1 << n
    obs = (Obs * count)()
    probs = np.empty(count * dim)
    vals = n - 5
    corr = np.arange(1, count * vals + 1, dtype=np.float64) / 7
    for j in range(count):
        x = _state(n, 10 + j)
        probs[j * dim:(j + 1) * dim] = x
        obs[j].n = n
        for b in range(n):
            obs[j].y[b] = 0.1 * (j + 1) + 0.01 * b
    s = Snaps(n, dim, 1, count, count, obs, _dp(probs), _dp(corr), None)
    prb = tmp_path / "o_prb.txt"
    host.me_write_prb_txt(str(prb).encode(), C.byref(s), 0.5)
    lines = prb.read_text().splitlines()
    assert len(lines) == count
    assert lines[1].startswith("0.500000, ")
    assert [float(v) for v in lines[2].split(",")[1:]] == pytest.approx(probs[2 * dim:], abs=5e-7)
    host.me_write_exp_timed(str(tmp_path / "o").encode(), C.byref(s), 0.5)
    rows = (tmp_path / "o_exp_timed.txt").read_text().splitlines()
    assert rows[2] == "1.000000, " + ", ".join("%f" % (0.3 + 0.01 * b) for b in range(n - 1, -1, -1))
    host.me_write_highcorr_timed(str(tmp_path / "o").encode(), C.byref(s), 0.5)
    rows = [r.split() for r in (tmp_path / "o_highcorr_timed").read_text().splitlines()]
    assert [r[0] for r in rows] == ["0.000000", "0.500000", "1.000000"]
    assert [float(r[1]) for r in rows] == pytest.approx(corr, rel=1e-6)
    # without snapshots the probability file is empty, as the reference leaves it
    host.me_write_prb_txt(str(tmp_path / "e_prb.txt").encode(), None, 0.5)
    assert (tmp_path / "e_prb.txt").read_text() == ""


@pytest.fixture(scope="module")
def warm(tmp_path_factory):
    import tasep_b200 as T
    out = tmp_path_factory.mktemp("warm") / "libmewarm.so"
    subprocess.run(["gcc", "-std=c99", "-O2", "-shared", "-fPIC", "-D_DEFAULT_SOURCE", "-I", HOST, "-I",
                    os.path.join(ROOT, "include"), os.path.join(HOST, "me_warm.c"), "-L", os.path.dirname(T.LIB_PATH),
                    "-ltasep_cuda", "-Wl,-rpath," + os.path.dirname(T.LIB_PATH), "-lm", "-o", str(out)], check=True)
    L = C.CDLL(str(out))
    L.me_warm_params_load.argtypes = [C.c_char_p, C.POINTER(C.c_float)]
    L.me_warm_mean_field.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.me_warm_features.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_float)]
    return L


def test_drop_in_warm_start_inputs_match_the_python_driver(warm):
    """--init learned builds the same network inputs as tasep_b200.warmstart and
    reads the shipped parameters."""
    from tasep_b200 import warmstart as ws
    for n, seed in ((12, 1), (20, 2)):
        r = ws.sample_rates(n, 1, np.random.default_rng(seed))[0]
        mf = np.empty(n)
        warm.me_warm_mean_field(n, _dp(r), _dp(mf))
        assert np.array_equal(mf, ws.mean_field_profile(r))
        f = np.empty((n, 16), dtype=np.float32)
        warm.me_warm_features(n, _dp(r), _dp(mf), f.ctypes.data_as(C.POINTER(C.c_float)))
        assert np.array_equal(f, ws.site_features(r))
    p = np.empty(9538, dtype=np.float32)
    assert warm.me_warm_params_load(ws.PRETRAINED.encode(), p.ctypes.data_as(C.POINTER(C.c_float))) == 0
    assert np.array_equal(p, np.load(ws.PRETRAINED))
    assert warm.me_warm_params_load(b"/nonexistent.npy", p.ctypes.data_as(C.POINTER(C.c_float))) == -1
