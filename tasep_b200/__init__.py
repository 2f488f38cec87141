"""tasep_b200 - B200 (sm_100a) TASEP master-equation integrator.

Python view of the C ABI in ``include/tasep.h`` (``libtasep_cuda.so``), used
by the tests and ``bench.py``.  The drop-in replacement for the reference's
``bin/masterEquation`` is the C program ``tasep_b200/bin/masterEquation``
built from ``tasep_b200/host``.  There is no CPU fallback: when the CUDA
library is missing every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libtasep_cuda.so")
CLI_PATH = os.path.join(PKG, "bin", "masterEquation")
INCLUDE = os.path.join(os.path.dirname(PKG), "include", "tasep.h")

INTEGRATOR_REF, INTEGRATOR_RK4 = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
INIT_UNIFORM, INIT_EMPTY = 0, 1
L2_OWN_FIRST, L2_DEMOTE, L2_FAR_FIRST = 1, 2, 4
FUN_SIN, FUN_COS, FUN_LIN = 0, 1, 2
MAX_N = 33

STATUS = {0: "OK", 1: "INVALID", 2: "NOMEM", 3: "CUDA", 4: "NODEV", 5: "TIMEOUT", 6: "UNSUPPORTED"}

# every symbol include/tasep.h declares
EXPORTS = (
    "tasep_meq_create", "tasep_meq_destroy", "tasep_meq_set_rates", "tasep_meq_set_timevar",
    "tasep_meq_clear_timevar", "tasep_meq_init", "tasep_meq_load", "tasep_meq_run",
    "tasep_meq_enqueue_steps", "tasep_meq_synchronize", "tasep_meq_store", "tasep_meq_observables",
    "tasep_meq_stream", "tasep_meq_profile", "tasep_meq_profile_read", "tasep_apply_device",
    "tasep_step_ref_device", "tasep_last_error", "tasep_abi_version", "tasep_meq_footprint",
    "tasep_step_ref_device_noalloc", "tasep_batch_create", "tasep_batch_destroy", "tasep_batch_set_rates",
    "tasep_batch_init", "tasep_batch_load", "tasep_batch_run", "tasep_batch_store", "tasep_batch_densities",
    "tasep_mlp_create", "tasep_mlp_destroy", "tasep_mlp_set_params", "tasep_mlp_get_params", "tasep_mlp_loss_grad",
    "tasep_mlp_train", "tasep_mlp_predict", "tasep_meq_init_pair_markov", "tasep_meq_run_snapshots",
    "tasep_meq_set_cache_policy", "tasep_meq_get_cache_policy", "tasep_test_inject_wait_expiry",
    "tasep_batch_last_config", "tasep_meq_run_stream", "tasep_test_div6", "tasep_mean_field_profile",
)


class TasepError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"tasep {STATUS.get(status, status)}: {msg}")
        self.status = status


class _Cfg(C.Structure):
    _fields_ = [("n", C.c_int), ("integrator", C.c_int), ("precision", C.c_int), ("device", C.c_int),
                ("stream", C.c_void_p)]


class _RunCfg(C.Structure):
    _fields_ = [("t0", C.c_double), ("h", C.c_double), ("steps", C.c_uint64), ("stop_tol", C.c_double),
                ("stop_count", C.c_int), ("exit_rule", C.c_int)]


class RunResult(C.Structure):
    _fields_ = [("steps_done", C.c_uint64), ("steps_at_stop", C.c_uint64), ("early_stop", C.c_int),
                ("converged", C.c_int), ("last_checksum", C.c_double), ("t_end", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_dp = C.POINTER(C.c_double)


def lib():
    """Load libtasep_cuda.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library missing: {LIB_PATH} (build with make -C tasep_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        H = C.c_void_p
        L.tasep_meq_create.argtypes = [C.POINTER(_Cfg), C.POINTER(H)]
        L.tasep_meq_destroy.argtypes = [H]
        L.tasep_meq_set_rates.argtypes = [H, _dp]
        L.tasep_meq_set_timevar.argtypes = [H, C.POINTER(C.c_int), _dp, _dp, _dp, _dp]
        L.tasep_meq_clear_timevar.argtypes = [H]
        L.tasep_meq_init.argtypes = [H, C.c_int]
        L.tasep_meq_load.argtypes = [H, _dp]
        L.tasep_meq_run.argtypes = [H, C.POINTER(_RunCfg), C.POINTER(RunResult)]
        L.tasep_meq_enqueue_steps.argtypes = [H, C.c_double, C.c_double, C.c_uint64]
        L.tasep_meq_synchronize.argtypes = [H]
        L.tasep_meq_store.argtypes = [H, _dp, C.c_uint64, C.c_uint64]
        L.tasep_meq_observables.argtypes = [H, _dp, _dp, _dp, _dp, _dp]
        L.tasep_meq_stream.argtypes = [H]
        L.tasep_meq_stream.restype = C.c_void_p
        L.tasep_meq_profile.argtypes = [H, C.c_int]
        L.tasep_meq_profile_read.argtypes = [H, C.POINTER(C.c_char_p), _dp, C.POINTER(C.c_uint64), C.c_int,
                                             C.POINTER(C.c_int)]
        L.tasep_apply_device.argtypes = [C.c_int, _dp, C.c_void_p, C.c_void_p, C.c_void_p]
        L.tasep_step_ref_device.argtypes = [C.c_int, _dp, C.c_double, C.c_void_p, C.c_void_p, _dp, C.c_void_p]
        L.tasep_step_ref_device_noalloc.argtypes = [C.c_int, _dp, C.c_double, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_void_p]
        L.tasep_last_error.restype = C.c_char_p
        L.tasep_abi_version.restype = C.c_int
        L.tasep_meq_footprint.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
        L.tasep_meq_footprint.restype = C.c_uint64
        L.tasep_meq_set_cache_policy.argtypes = [H, C.c_int, C.c_int]
        L.tasep_meq_get_cache_policy.argtypes = [H, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.tasep_test_inject_wait_expiry.argtypes = [C.c_uint64, C.c_int]
        L.tasep_test_div6.argtypes = [_dp, _dp, C.c_uint64]
        _lib = L
    return _lib


def _check(st):
    if st != 0:
        raise TasepError(st, lib().tasep_last_error().decode())


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def inject_wait_expiry(wait_limit_ns=0, skip_partner_copy=-1):
    """Test hook: bounded device waits give up after wait_limit_ns and the first
    CTA leaves out one partner copy (see include/tasep.h); (0, -1) turns it off."""
    _check(lib().tasep_test_inject_wait_expiry(int(wait_limit_ns), int(skip_partner_copy)))


def div6(x):
    """Test entry: x / 6 as the device steps compute it (see include/tasep.h)."""
    x = _f64(x).ravel()
    out = np.empty_like(x)
    _check(lib().tasep_test_div6(x.ctypes.data_as(_dp), out.ctypes.data_as(_dp), x.size))
    return out


def footprint(n, integrator=INTEGRATOR_RK4, precision=PRECISION_FP64, timevar=False):
    return int(lib().tasep_meq_footprint(n, integrator, precision, int(timevar)))


class Meq:
    """One master-equation system on one GPU (mirrors the tasep_meq_* calls)."""

    def __init__(self, n, integrator=INTEGRATOR_REF, precision=PRECISION_FP64, device=-1, stream=None):
        self.n = n
        self._h = C.c_void_p()
        cfg = _Cfg(n, integrator, precision, device, stream)
        _check(lib().tasep_meq_create(C.byref(cfg), C.byref(self._h)))

    def close(self):
        if self._h:
            lib().tasep_meq_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_rates(self, rates):
        r = _f64(rates)
        assert r.shape == (self.n + 1,)
        _check(lib().tasep_meq_set_rates(self._h, r.ctypes.data_as(_dp)))

    def set_timevar(self, type, amplitude, period, offset, constant):
        ty = np.ascontiguousarray(type, dtype=np.int32)
        arrs = [_f64(a) for a in (amplitude, period, offset, constant)]
        _check(lib().tasep_meq_set_timevar(self._h, ty.ctypes.data_as(C.POINTER(C.c_int)),
                                           *[a.ctypes.data_as(_dp) for a in arrs]))

    def clear_timevar(self):
        _check(lib().tasep_meq_clear_timevar(self._h))

    def init(self, kind=INIT_EMPTY):
        _check(lib().tasep_meq_init(self._h, kind))

    def load(self, x):
        x = _f64(x)
        assert x.shape == (1 << self.n,)
        _check(lib().tasep_meq_load(self._h, x.ctypes.data_as(_dp)))

    def run(self, h, steps, t0=0.0, stop_tol=1e-10, stop_count=100, exit_rule=True):
        rc = _RunCfg(t0, h, steps, stop_tol, stop_count, int(bool(exit_rule)))
        res = RunResult()
        _check(lib().tasep_meq_run(self._h, C.byref(rc), C.byref(res)))
        return res.as_dict()

    def run_snapshots(self, h, steps, every, fn, t0=0.0, stop_tol=1e-10, stop_count=100, exit_rule=True):
        """run() calling fn(self, step, t) after every step whose index is a multiple of `every`."""
        L = lib()
        hook_t = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_double, C.c_void_p)
        L.tasep_meq_run_snapshots.argtypes = [C.c_void_p, C.POINTER(_RunCfg), C.c_uint64, hook_t, C.c_void_p,
                                              C.POINTER(RunResult)]
        errors = []

        def hook(_h, step, t, _u):
            try:
                fn(self, step, t)
            except Exception as e:  # an exception cannot cross the C frame
                errors.append(e)

        cb = hook_t(hook)
        rc = _RunCfg(t0, h, steps, stop_tol, stop_count, int(bool(exit_rule)))
        res = RunResult()
        _check(L.tasep_meq_run_snapshots(self._h, C.byref(rc), every, cb, None, C.byref(res)))
        if errors:
            raise errors[0]
        return res.as_dict()

    def run_stream(self, h, steps, every, fn, with_probs=False, t0=0.0, stop_tol=1e-10, stop_count=100,
                   exit_rule=True):
        """run() with snapshots that do not stop the integration: fn(step, t, obs, probs) for every step
        whose index is a multiple of `every`, in step order, with obs a dict of copies of rho (bit
        order), cov and mul (site order) and window4 ((n-3, 16), n >= 4), and probs a copy of the
        2^n probabilities (None unless with_probs)."""
        L = lib()
        P = C.POINTER(C.c_double)
        hook_t = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_double, P, P, P, P, P, C.c_void_p)
        L.tasep_meq_run_stream.argtypes = [C.c_void_p, C.POINTER(_RunCfg), C.c_uint64, C.c_int, hook_t,
                                           C.c_void_p, C.POINTER(RunResult)]
        n, errors = self.n, []

        def arr(p, k):
            return np.ctypeslib.as_array(p, (k,)).copy() if p else None

        def hook(_h, step, t, rho, cov, mul, w4, probs, _u):
            try:
                obs = {"rho": arr(rho, n), "cov": arr(cov, n * n).reshape(n, n),
                       "mul": arr(mul, n * n).reshape(n, n)}
                if n >= 4:
                    obs["window4"] = arr(w4, (n - 3) * 16).reshape(n - 3, 16)
                fn(step, t, obs, arr(probs, 1 << n))
            except Exception as e:  # an exception cannot cross the C frame
                errors.append(e)

        cb = hook_t(hook)
        rc = _RunCfg(t0, h, steps, stop_tol, stop_count, int(bool(exit_rule)))
        res = RunResult()
        _check(L.tasep_meq_run_stream(self._h, C.byref(rc), every, int(bool(with_probs)), cb, None,
                                      C.byref(res)))
        if errors:
            raise errors[0]
        return res.as_dict()

    def enqueue_steps(self, h, steps, t0=0.0):
        _check(lib().tasep_meq_enqueue_steps(self._h, t0, h, steps))

    def synchronize(self):
        _check(lib().tasep_meq_synchronize(self._h))

    def store(self, out=None, offset=0, count=None):
        if count is None:
            count = (1 << self.n) - offset
        if out is None:
            out = np.empty(count)
        _check(lib().tasep_meq_store(self._h, out.ctypes.data_as(_dp), offset, count))
        return out

    def observables(self):
        n = self.n
        rho, cov, mul = np.empty(n), np.empty(n * n), np.empty(n * n)
        w4 = np.empty(max(n - 3, 0) * 16 or 1)
        mass = np.empty(1)
        _check(lib().tasep_meq_observables(self._h, rho.ctypes.data_as(_dp), cov.ctypes.data_as(_dp),
                                           mul.ctypes.data_as(_dp), w4.ctypes.data_as(_dp),
                                           mass.ctypes.data_as(_dp)))
        return {"rho": rho, "cov": cov.reshape(n, n), "mul": mul.reshape(n, n),
                "window4": w4[:max(n - 3, 0) * 16].reshape(-1, 16), "mass": float(mass[0])}

    @property
    def stream(self):
        return lib().tasep_meq_stream(self._h)

    def profile(self, enable=True):
        _check(lib().tasep_meq_profile(self._h, int(enable)))

    def set_cache_policy(self, near_bits, flags):
        """L2 policy of the generator sweep (speed only; results do not depend on it)."""
        _check(lib().tasep_meq_set_cache_policy(self._h, near_bits, flags))

    def cache_policy(self):
        a, b = C.c_int(0), C.c_int(0)
        _check(lib().tasep_meq_get_cache_policy(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def profile_read(self):
        cap = 16
        names = (C.c_char_p * cap)()
        ms = np.zeros(cap)
        cnt = (C.c_uint64 * cap)()
        k = C.c_int(0)
        _check(lib().tasep_meq_profile_read(self._h, names, ms.ctypes.data_as(_dp), cnt, cap, C.byref(k)))
        return {names[i].decode(): (float(ms[i]), int(cnt[i])) for i in range(min(k.value, cap))}


class Batch:
    """nsys independent systems of length n in one sweep (tasep_batch_* calls)."""

    def __init__(self, n, nsys, precision=PRECISION_FP64, device=-1, stream=None):
        L = lib()
        H = C.c_void_p
        if not getattr(L, "_batch_types", False):
            L.tasep_batch_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.POINTER(H)]
            L.tasep_batch_destroy.argtypes = [H]
            L.tasep_batch_set_rates.argtypes = [H, _dp]
            L.tasep_batch_init.argtypes = [H, C.c_int]
            L.tasep_batch_load.argtypes = [H, _dp]
            L.tasep_batch_run.argtypes = [H, C.POINTER(_RunCfg), C.c_int, C.POINTER(RunResult), C.POINTER(C.c_int)]
            L.tasep_batch_store.argtypes = [H, C.c_int, _dp]
            L.tasep_batch_densities.argtypes = [H, _dp]
            L.tasep_batch_last_config.argtypes = [H, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
            L._batch_types = True
        self.n, self.nsys = n, nsys
        self._h = H()
        _check(L.tasep_batch_create(n, nsys, precision, device, stream, C.byref(self._h)))

    def close(self):
        if self._h:
            lib().tasep_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_rates(self, rates):
        r = _f64(rates).reshape(self.nsys, self.n + 1)
        _check(lib().tasep_batch_set_rates(self._h, r.ctypes.data_as(_dp)))

    def init(self, kind=INIT_EMPTY):
        _check(lib().tasep_batch_init(self._h, kind))

    def load(self, x):
        x = _f64(x).reshape(self.nsys, 1 << self.n)
        _check(lib().tasep_batch_load(self._h, x.ctypes.data_as(_dp)))

    def run(self, h, steps, stop_tol=1e-10, stop_count=100, exit_rule=True, schedule=-1, t0=0.0):
        rc = _RunCfg(t0, h, steps, stop_tol, stop_count, int(bool(exit_rule)))
        res = (RunResult * self.nsys)()
        used = C.c_int(-1)
        _check(lib().tasep_batch_run(self._h, C.byref(rc), schedule, res, C.byref(used)))
        return [r.as_dict() for r in res], used.value

    def store(self, sys):
        out = np.empty(1 << self.n)
        _check(lib().tasep_batch_store(self._h, sys, out.ctypes.data_as(_dp)))
        return out

    def last_config(self):
        """(schedule, states per CTA, CTAs per system) of the last run."""
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        _check(lib().tasep_batch_last_config(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def densities(self):
        rho = np.empty((self.nsys, self.n))
        _check(lib().tasep_batch_densities(self._h, rho.ctypes.data_as(_dp)))
        return rho


MLP_IN, MLP_OUT, MLP_PARAMS = 16, 2, 9538
_fp = C.POINTER(C.c_float)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Mlp:
    """The per-site surrogate network, trained and evaluated on the GPU."""

    def __init__(self, seed=0, device=-1):
        L = lib()
        H = C.c_void_p
        if not getattr(L, "_mlp_types", False):
            L.tasep_mlp_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(H)]
            L.tasep_mlp_destroy.argtypes = [H]
            L.tasep_mlp_set_params.argtypes = [H, _fp]
            L.tasep_mlp_get_params.argtypes = [H, _fp]
            L.tasep_mlp_loss_grad.argtypes = [H, _fp, _fp, C.c_int, _fp, _fp, _fp]
            L.tasep_mlp_train.argtypes = [H, _fp, _fp, C.c_int, _fp, C.c_int, C.c_int, C.c_float, C.c_uint64, _fp]
            L.tasep_mlp_predict.argtypes = [H, _fp, C.c_int, _fp]
            L.tasep_meq_init_pair_markov.argtypes = [H, _dp, _dp]
            L._mlp_types = True
        self._h = H()
        _check(L.tasep_mlp_create(device, seed, C.byref(self._h)))

    def close(self):
        if self._h:
            lib().tasep_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self):
        p = np.empty(MLP_PARAMS, dtype=np.float32)
        _check(lib().tasep_mlp_get_params(self._h, p.ctypes.data_as(_fp)))
        return p

    @params.setter
    def params(self, p):
        p = _f32(p)
        assert p.shape == (MLP_PARAMS,)
        _check(lib().tasep_mlp_set_params(self._h, p.ctypes.data_as(_fp)))

    def loss_grad(self, x, t, out_weights=(1.0, 1.0)):
        x, t, w = _f32(x), _f32(t), _f32(out_weights)
        loss = np.zeros(1, dtype=np.float32)
        g = np.empty(MLP_PARAMS, dtype=np.float32)
        _check(lib().tasep_mlp_loss_grad(self._h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), len(x),
                                         w.ctypes.data_as(_fp), loss.ctypes.data_as(_fp), g.ctypes.data_as(_fp)))
        return float(loss[0]), g

    def train(self, x, t, out_weights=(1.0, 1.0), epochs=100, batch=1024, lr=1e-3, seed=0):
        x, t, w = _f32(x), _f32(t), _f32(out_weights)
        losses = np.zeros(max(epochs, 1), dtype=np.float32)
        _check(lib().tasep_mlp_train(self._h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), len(x),
                                     w.ctypes.data_as(_fp), epochs, batch, lr, seed, losses.ctypes.data_as(_fp)))
        return losses[:epochs]

    def predict(self, x):
        x = _f32(x)
        y = np.empty((len(x), MLP_OUT), dtype=np.float32)
        _check(lib().tasep_mlp_predict(self._h, x.ctypes.data_as(_fp), len(x), y.ctypes.data_as(_fp)))
        return y


def init_pair_markov(meq, rho, cov):
    """Pair-Markov initial measure on a Meq handle; raises TasepError if infeasible."""
    L = lib()
    L.tasep_meq_init_pair_markov.argtypes = [C.c_void_p, _dp, _dp]
    r, c = _f64(rho), _f64(cov)
    _check(L.tasep_meq_init_pair_markov(meq._h, r.ctypes.data_as(_dp), c.ctypes.data_as(_dp)))


def apply_device(n, rates, x_ptr, y_ptr, stream=None):
    """y = M x on device pointers (ints)."""
    r = _f64(rates)
    _check(lib().tasep_apply_device(n, r.ctypes.data_as(_dp), x_ptr, y_ptr, stream))


def step_ref_device(n, rates, h, x_ptr, out_ptr, stream=None):
    """One reference step on device pointers; returns the L1 norm of the increment."""
    r = _f64(rates)
    cs = C.c_double(0.0)
    _check(lib().tasep_step_ref_device(n, r.ctypes.data_as(_dp), h, x_ptr, out_ptr, C.byref(cs), stream))
    return cs.value


def step_ref_device_noalloc(n, rates, h, x_ptr, out_ptr, checksum_ptr=None, stream=None):
    """One reference step on device pointers using only the library's static
    scratch (no device allocation); the L1 norm goes to checksum_ptr (device)."""
    r = _f64(rates)
    _check(lib().tasep_step_ref_device_noalloc(n, r.ctypes.data_as(_dp), h, x_ptr, out_ptr, checksum_ptr,
                                               stream))
