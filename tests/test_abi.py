"""The C ABI without a GPU: the library loads, exports every entry point that
include/tasep.h declares, and fails cleanly (status codes, no crash) when no
device is present."""
import ctypes as C
import os
import re

import pytest

import tasep_b200 as T

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "tasep.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tasep_[a-z0-9_]+)\s*\(", text)))


def test_header_declarations_are_all_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = C.CDLL(T.LIB_PATH)
    missing = [nm for nm in names if not hasattr(lib, nm)]
    assert not missing, missing
    assert set(names) == set(T.EXPORTS)


def test_abi_version_and_footprint():
    L = T.lib()
    assert L.tasep_abi_version() == 1
    N = 1 << 28
    assert T.footprint(28, T.INTEGRATOR_RK4, T.PRECISION_FP64) == 32 * N
    assert T.footprint(28, T.INTEGRATOR_REF, T.PRECISION_FP64) == 16 * N
    assert T.footprint(33, T.INTEGRATOR_RK4, T.PRECISION_MIXED) == 20 * (1 << 33)  # 171.8 GB < 180 GB
    assert T.footprint(0, 0, 0) == 0 and T.footprint(34, 0, 0) == 0


def test_invalid_arguments_are_rejected_before_touching_a_device():
    with pytest.raises(T.TasepError) as e:
        T.Meq(0)
    assert e.value.status == 1
    with pytest.raises(T.TasepError) as e:
        T.Meq(40)
    assert e.value.status == 1
    with pytest.raises(T.TasepError) as e:
        T.Meq(10, T.INTEGRATOR_REF, T.PRECISION_MIXED)
    assert e.value.status == 6  # mixed precision is for RK4 only


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and __import__("torch").cuda.is_available(),
                    reason="a GPU is present")
def test_no_device_reports_nodev():
    with pytest.raises(T.TasepError) as e:
        T.Meq(10)
    assert e.value.status == 4
    assert "no CUDA device" in str(e.value)


def test_sweep_and_warm_start_entry_points_validate_arguments():
    for n, nsys in ((11, 4), (25, 4), (16, 0)):
        with pytest.raises(T.TasepError) as e:
            T.Batch(n, nsys)
        assert e.value.status == 1
    L = T.lib()
    assert L.tasep_mlp_create(0, 1, None) == 1
    assert L.tasep_mlp_destroy(None) == 0
    assert L.tasep_meq_init_pair_markov(None, None, None) == 1
    hook_t = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_double, C.c_void_p)
    L.tasep_meq_run_snapshots.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, hook_t, C.c_void_p, C.c_void_p]
    assert L.tasep_meq_run_snapshots(None, None, 1, hook_t(lambda *a: None), None, None) == 1
    P = C.POINTER(C.c_double)
    stream_t = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_double, P, P, P, P, P, C.c_void_p)
    L.tasep_meq_run_stream.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, stream_t, C.c_void_p,
                                       C.c_void_p]
    assert L.tasep_meq_run_stream(None, None, 1, 0, stream_t(lambda *a: None), None, None) == 1
    assert b"" != L.tasep_last_error()


def test_cache_policy_and_test_hook_validate_without_a_device():
    L = T.lib()
    assert L.tasep_meq_set_cache_policy(None, 12, 0) == 1
    assert L.tasep_meq_get_cache_policy(None, None, None) == 1
    with pytest.raises(T.TasepError) as e:
        T.inject_wait_expiry(0, -2)
    assert e.value.status == 1
    T.inject_wait_expiry(0, -1)  # off: accepted without a device
