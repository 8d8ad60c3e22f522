"""ocean_symbolic_noalloc: exact per-row output counts without any allocation
by the library, for callers that own all device memory themselves (an
application arena or caching allocator) or may not call cudaMalloc in steady
state. Its scratch is a fixed device array inside the library, so it checks:
  * two calls in a row through the C ABI (a different matrix each time, so the
    second call must not see the first call's scratch contents) give exactly
    the counts of the regular entry point ocean_symbolic;
  * an A with more rows than the fixed scratch allows is refused with
    OCEAN_ERR_INVALID.
This file is collected last on purpose (name order)."""
import ctypes

import numpy as np
import pytest

from research_b200 import matrices as M
from research_b200.ocean import CsrView, DeviceCSR, SpGEMM, lib

pytestmark = pytest.mark.gpu

MAX_ROWS = 131072


def noalloc_counts(dA, dB):
    import torch
    out = torch.full((dA.rows,), -1, dtype=torch.int32, device="cuda")
    av, bv = dA.view(), dB.view()
    rc = lib().ocean_symbolic_noalloc(ctypes.byref(av), ctypes.byref(bv), out.data_ptr(), None)
    assert rc == 0, lib().ocean_last_error()
    return out.cpu().numpy().view(np.uint32)


def test_noalloc_matches_regular_entry_point_twice():
    # first a skewed R-MAT (every class, bitmap rows included), then a smaller
    # uniform matrix: the second call reuses the scratch the first one filled
    cases = [M.rmat(17, 16, seed=31), M.uniform_random(40000, 12, seed=32)]
    g = SpGEMM()
    for A in cases:
        dA = DeviceCSR.from_host(A)
        got = noalloc_counts(dA, dA)
        want = g.symbolic(dA, dA).cpu().numpy().view(np.uint32)
        assert got.shape == want.shape
        assert np.array_equal(got, want)


def test_noalloc_rejects_more_rows_than_scratch():
    A = M.uniform_random(MAX_ROWS + 1, 1, seed=33)
    dA = DeviceCSR.from_host(A)
    import torch
    out = torch.empty(A.rows, dtype=torch.int32, device="cuda")
    av = dA.view()
    rc = lib().ocean_symbolic_noalloc(ctypes.byref(av), ctypes.byref(av), out.data_ptr(), None)
    assert rc == 4
    assert b"more than the fixed scratch allows" in lib().ocean_last_error()
