"""The REF and time-variant steps divide (k1 + 2 k2 + 2 k3 + k4) by 6 without
a division instruction sequence (Markstein's correction step, proof beside
div6_rn in meq_common.cuh).  The device result must equal the correctly
rounded IEEE quotient that the reference's `/ 6` gives on the host, bit for
bit, over the whole double range: every binade, the values the step produces
(k + 2k + 2k + k sums), the edges of the fast path and the special values."""
import numpy as np
import pytest

import tasep_b200 as T

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_div6_every_binade_bit_exact():
    rng = np.random.default_rng(6)
    # random significands in every binade from the subnormals to 2^1023
    bits = rng.integers(0, 1 << 52, size=1 << 22, dtype=np.uint64)
    exps = rng.integers(0, 2047, size=bits.size, dtype=np.uint64)  # 0 = subnormal
    x = ((exps << np.uint64(52)) | bits).view(np.float64)
    x = np.concatenate([x, -x])
    y = T.div6(x)
    with np.errstate(over="ignore", under="ignore", invalid="ignore"):
        ref = x / 6.0
    assert _same(y, ref)


def test_div6_step_sums_and_edges_bit_exact():
    rng = np.random.default_rng(7)
    # the sums the step forms: kv = h * (M x)_i, then ((kv + 2kv) + 2kv) + kv
    kv = rng.standard_normal(1 << 21) * np.exp2(rng.integers(-1000, 5, size=1 << 21))
    k2 = 2.0 * kv
    s = ((kv + k2) + k2) + kv
    # multiples of 6 and their neighbours, powers of two, the fast path's edges
    m6 = 6.0 * rng.integers(1, 1 << 50, size=1 << 16).astype(np.float64)
    p2 = np.exp2(np.arange(-1074, 1024, dtype=np.float64))
    edges = np.array([2.0 ** -900, 2.0 ** 1000], dtype=np.float64)
    near = np.concatenate([np.nextafter(v, np.inf) for v in (m6, p2, edges)] +
                          [np.nextafter(v, -np.inf) for v in (m6, p2, edges)])
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, -5e-324, 6.0, 1.0, 1e308])
    x = np.concatenate([s, m6, p2, edges, near, special])
    x = np.concatenate([x, -x])
    y = T.div6(x)
    with np.errstate(over="ignore", under="ignore", invalid="ignore"):
        ref = x / 6.0
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(y), nan)
    assert _same(y[~nan], ref[~nan])
