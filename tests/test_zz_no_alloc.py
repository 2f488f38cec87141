"""The allocation-free reference step against the allocating one.

tasep_step_ref_device_noalloc serves callers that cannot call cudaMalloc (a
host program whose device memory all comes from its own pool allocator, or a
loop that cannot pay for the synchronisation an allocation may cause).  It
keeps its scratch in a fixed array in the library's device image.  Here it
must give the same next state and the same L1 norm as tasep_step_ref_device
(bit for bit, the bar the reference step is held to everywhere), on two
calls in a row, so the second call also shows that the array's leftovers
from the first call are cleared.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import numpy as np
import pytest

import tasep_b200 as T

pytestmark = pytest.mark.gpu


def rates_for(n, seed):
    rng = np.random.default_rng(seed)
    r = np.empty(n + 1)
    r[0], r[n] = rng.uniform(0.1, 1.0, 2)
    r[1:n] = np.clip(rng.lognormal(0.0, 0.5, n - 1), 0.1, 5.0)
    return r


@pytest.mark.parametrize("n", [9, 14, 22])
def test_noalloc_step_matches_allocating_step(n):
    import torch
    assert torch.cuda.is_available(), "CUDA device required"
    r = rates_for(n, 40 + n)
    h = 0.01
    x = torch.from_numpy(np.random.default_rng(n).random(1 << n)).cuda()
    x /= x.sum()
    ref_out = torch.empty_like(x)
    ref_cs = T.step_ref_device(n, r, h, x.data_ptr(), ref_out.data_ptr())
    for _ in range(2):
        out = torch.full_like(x, float("nan"))
        cs = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        T.step_ref_device_noalloc(n, r, h, x.data_ptr(), out.data_ptr(), cs.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(out, ref_out)
        assert cs.item() == ref_cs


def test_noalloc_step_marks_an_expired_wait_with_nan():
    """The allocation-free step keeps its status in the shared static array,
    out of the caller's reach; a bounded wait that expired must still be
    visible, as a NaN norm in checksum_dev.  The next call, with the test hook
    off, must clear that state and agree with the allocating step again."""
    import torch
    assert torch.cuda.is_available(), "CUDA device required"
    n = 14
    r = rates_for(n, 61)
    x = torch.from_numpy(np.random.default_rng(61).random(1 << n)).cuda()
    out = torch.empty_like(x)
    cs = torch.zeros(1, dtype=torch.float64, device="cuda")
    try:
        T.inject_wait_expiry(1_000_000, 0)
        T.step_ref_device_noalloc(n, r, 0.01, x.data_ptr(), out.data_ptr(), cs.data_ptr())
        torch.cuda.synchronize()
    finally:
        T.inject_wait_expiry(0, -1)
    assert np.isnan(cs.item())
    ref_out = torch.empty_like(x)
    ref_cs = T.step_ref_device(n, r, 0.01, x.data_ptr(), ref_out.data_ptr())
    T.step_ref_device_noalloc(n, r, 0.01, x.data_ptr(), out.data_ptr(), cs.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(out, ref_out)
    assert cs.item() == ref_cs
