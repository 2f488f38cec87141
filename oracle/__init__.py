"""CPU oracle for the TASEP master-equation integrator.

TEST INFRASTRUCTURE ONLY.  This package is the checker: tests/,
``__graft_entry__.smoke()`` and ``bench.py`` (its cpu_baseline leg and the
``--impl reference`` arm) may load it.  The product (``tasep_b200``) never
imports it.

Two back ends:

* ``liboracle.so`` - the project's plain-C restatement of the reference
  algorithm (``oracle/tasep_oracle.c``; each function cites the reference
  file:line it follows).
* ``_ref/libtasep_ref.so`` - the reference's own ``src/lib/*.c`` compiled in
  place plus a driver loop (``oracle/ref_harness.c``).  Built only where the
  reference sources exist; the built file travels with the repository.

``mpa`` holds an exact-rational restatement of the reference's matrix-product
steady state (``src/steadystates_gmp.c``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtasep_ref.so")
REF_BIN = os.path.join(HERE, "_ref", "masterEquation")

INT_REF, INT_RK4 = 0, 1
INIT_UNIFORM, INIT_EMPTY = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _RunCfg(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("integrator", C.c_int), ("init", C.c_int),
        ("x0", _dp), ("rates", _dp), ("timevar", C.c_int), ("tv_type", _ip),
        ("tv_amplitude", _dp), ("tv_period", _dp), ("tv_offset", _dp), ("tv_constant", _dp),
        ("t0", C.c_double), ("h", C.c_double), ("steps", C.c_uint64),
        ("stop_tol", C.c_double), ("stop_count", C.c_int), ("exit_rule", C.c_int),
    ]


class RunResult(C.Structure):
    _fields_ = [
        ("steps_done", C.c_uint64), ("steps_at_stop", C.c_uint64), ("early_stop", C.c_int),
        ("last_checksum", C.c_double), ("t_end", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_ref = None


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def lib():
    """Load liboracle.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle not built: {ORACLE_SO} missing (run make -C oracle oracle)")
        L = C.CDLL(ORACLE_SO)
        L.orc_apply.argtypes = [C.c_int, _dp, _dp, _dp]
        L.orc_gen_row.argtypes = [C.c_int, C.c_uint64, _dp, _dp, C.POINTER(C.c_uint64)]
        L.orc_gen_row.restype = C.c_int
        L.orc_timevar_rates.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, _ip, _dp, _dp]
        L.orc_step_ref.argtypes = [C.c_int, _dp, C.c_double, _dp, _dp]
        L.orc_step_ref.restype = C.c_double
        L.orc_step_rk4.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_double, _dp, _dp]
        L.orc_step_rk4.restype = C.c_double
        L.orc_run.argtypes = [C.POINTER(_RunCfg), _dp, C.POINTER(RunResult)]
        L.orc_densities.argtypes = [C.c_int, _dp, _dp]
        L.orc_covariance.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
        for f in ("orc_high_order_corr", "orc_error_guess", "orc_pf_approx", "orc_point_func"):
            fn = getattr(L, f)
            fn.argtypes = [_dp, C.c_uint64, C.c_uint64, C.c_int, C.c_int]
            fn.restype = C.c_double
        L.orc_window4.argtypes = [C.c_int, _dp, _dp]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """Load the reference-linked harness (raises if it was not built)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"reference harness not built: {REF_SO} missing")
        L = C.CDLL(REF_SO)
        L.refh_run.argtypes = [
            C.c_int, _dp, C.c_double, C.c_double, C.c_uint64, C.c_double, C.c_int, C.c_int,
            C.c_int, C.c_int, _ip, _dp, _dp, _dp, _dp, C.c_int, _dp, C.POINTER(RunResult)]
        L.refh_time_sample.argtypes = [C.c_int, C.c_uint64, _dp, C.c_double, C.c_int, C.c_int,
                                       C.POINTER(C.c_uint64)]
        L.refh_time_sample.restype = C.c_double
        L.refh_gencrs.argtypes = [C.c_int, C.c_uint64, _dp, C.POINTER(C.c_uint64), _dp,
                                  C.POINTER(C.c_uint64)]
        L.refh_gencrs.restype = C.c_uint64
        L.refh_max_threads.restype = C.c_int
        _ref = L
    return _ref


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def apply(n, rates, x):
    """y = M x, rows summed in the reference order."""
    rates, x = _f64(rates), _f64(x)
    y = np.empty(1 << n)
    lib().orc_apply(n, _d(rates), _d(x), _d(y))
    return y


def gen_row(n, i, rates):
    rates = _f64(rates)
    val = np.zeros(72)
    col = (C.c_uint64 * 72)()
    c = lib().orc_gen_row(n, i, _d(rates), _d(val), col)
    return [int(col[j]) for j in range(c)], val[:c].copy()


def timevar_rates(t, tv):
    """Rates at time t from a dict(type, amplitude, period, offset, constant)."""
    ty = np.ascontiguousarray(tv["type"], dtype=np.int32)
    out = np.empty(len(ty))
    lib().orc_timevar_rates(len(ty), _d(_f64(tv["period"])), _d(_f64(tv["offset"])),
                            _d(_f64(tv["amplitude"])), t, ty.ctypes.data_as(_ip),
                            _d(_f64(tv["constant"])), _d(out))
    return out


def step_ref(n, rates, h, x):
    """One reference-compatible step in place; returns the L1 norm of the increment."""
    k = np.empty(1 << n)
    return lib().orc_step_ref(n, _d(_f64(rates)), h, _d(x), _d(k))


def step_rk4(n, r1, h, x, r2=None, r3=None, r4=None):
    s = np.empty(6 << n)
    r1 = _f64(r1)
    r2 = r1 if r2 is None else _f64(r2)
    r3 = r2 if r3 is None else _f64(r3)
    r4 = r1 if r4 is None else _f64(r4)
    return lib().orc_step_rk4(n, _d(r1), _d(r2), _d(r3), _d(r4), h, _d(x), _d(s))


def run(n, rates=None, h=0.01, steps=100, integrator=INT_REF, init=INIT_EMPTY, x0=None,
        stop_tol=1e-10, stop_count=100, exit_rule=True, t0=0.0, timevar=None):
    """Integrate with the reference loop and exit rule; returns (x, result-dict)."""
    cfg = _RunCfg()
    keep = []
    cfg.n, cfg.integrator, cfg.init = n, integrator, init
    if x0 is not None:
        x0 = _f64(x0)
        keep.append(x0)
        cfg.x0 = _d(x0)
    if rates is not None:
        rates = _f64(rates)
        keep.append(rates)
        cfg.rates = _d(rates)
    if timevar is not None:
        ty = np.ascontiguousarray(timevar["type"], dtype=np.int32)
        arrs = [_f64(timevar[k]) for k in ("amplitude", "period", "offset", "constant")]
        keep += [ty] + arrs
        cfg.timevar = 1
        cfg.tv_type = ty.ctypes.data_as(_ip)
        cfg.tv_amplitude, cfg.tv_period, cfg.tv_offset, cfg.tv_constant = [_d(a) for a in arrs]
    cfg.t0, cfg.h, cfg.steps = t0, h, steps
    cfg.stop_tol, cfg.stop_count, cfg.exit_rule = stop_tol, stop_count, int(bool(exit_rule))
    x = np.empty(1 << n)
    res = RunResult()
    if lib().orc_run(C.byref(cfg), _d(x), C.byref(res)) != 0:
        raise MemoryError("oracle run failed")
    return x, res.as_dict()


def densities(n, x):
    y = np.empty(n)
    lib().orc_densities(n, _d(_f64(x)), _d(y))
    return y


def covariance(n, x, y=None):
    """(cov, mul) n x n in site order, as the reference writes them."""
    x = _f64(x)
    if y is None:
        y = densities(n, x)
    cov = np.empty(n * n)
    mul = np.empty(n * n)
    lib().orc_covariance(n, _d(x), _d(_f64(y)), _d(cov), _d(mul))
    return cov.reshape(n, n), mul.reshape(n, n)


def window4(n, x):
    p4 = np.zeros(max(n - 3, 0) * 16)
    if n >= 4:
        lib().orc_window4(n, _d(_f64(x)), _d(p4))
    return p4.reshape(-1, 16)


def high_order_corr(x, key, key_size, offset):
    x = _f64(x)
    return lib().orc_high_order_corr(_d(x), len(x), key, key_size, offset)


def error_guess(x, key, key_size, offset):
    x = _f64(x)
    return lib().orc_error_guess(_d(x), len(x), key, key_size, offset)


def pf_approx(x, key, key_size, offset):
    x = _f64(x)
    return lib().orc_pf_approx(_d(x), len(x), key, key_size, offset)


def point_func(x, key, key_size, offset):
    x = _f64(x)
    return lib().orc_point_func(_d(x), len(x), key, key_size, offset)


def ref_run(n, rates, h=0.01, steps=100, init=INIT_EMPTY, stop_tol=1e-10, stop_count=100,
            use_csr=True, timevar=None, t0=0.0, nthreads=0):
    """Run the reference's compiled step code; returns (x, result-dict)."""
    rates = _f64(rates)
    x = np.empty(1 << n)
    res = RunResult()
    if timevar is not None:
        ty = np.ascontiguousarray(timevar["type"], dtype=np.int32)
        arrs = [_f64(timevar[k]) for k in ("amplitude", "period", "offset", "constant")]
        tvargs = [1, ty.ctypes.data_as(_ip)] + [_d(a) for a in arrs]
    else:
        tvargs = [0, None, None, None, None, None]
    ref().refh_run(n, _d(rates), t0, h, steps, stop_tol, stop_count, init, int(use_csr),
                   *tvargs, nthreads, _d(x), C.byref(res))
    return x, res.as_dict()


def ref_csr_matches_gencrs(n, rates):
    """True when the harness's parallel CSR builder reproduces gencrs exactly."""
    L = ref()
    L.refh_csr_matches_gencrs.argtypes = [C.c_int, _dp]
    return L.refh_csr_matches_gencrs(n, _d(_f64(rates))) == 1


def ref_time_full(n, rates, h=0.01, warm=1, reps=1, nthreads=0):
    """Seconds per reference -f step over all 2^n rows, set-up seconds and nnz."""
    L = ref()
    L.refh_time_full.argtypes = [C.c_int, _dp, C.c_double, C.c_int, C.c_int, C.c_int, _dp,
                                 C.POINTER(C.c_uint64)]
    L.refh_time_full.restype = C.c_double
    build, nnz = C.c_double(0.0), C.c_uint64(0)
    s = L.refh_time_full(n, _d(_f64(rates)), h, warm, reps, nthreads, C.byref(build), C.byref(nnz))
    return s, float(build.value), int(nnz.value)


def ref_time_sample(n, rows, rates, h=0.01, reps=1, nthreads=0):
    """Seconds per reference -f step over the first `rows` rows (and nnz)."""
    nnz = C.c_uint64(0)
    s = ref().refh_time_sample(n, rows, _d(_f64(rates)), h, reps, nthreads, C.byref(nnz))
    return s, int(nnz.value)
