"""ocean_symbolic_noalloc: exact per-row output counts without any allocation
by the library, for callers that own all device memory themselves (an
application arena or caching allocator) or may not call cudaMalloc in steady
state. Its scratch is a fixed device array inside the library, so it checks:
  * two calls in a row through the C ABI (a different matrix each time, so the
    second call must not see the first call's scratch contents) give exactly
    the counts of the regular entry point ocean_symbolic and of the CPU oracle,
    with 32- and with 64-bit row pointers;
  * a call after a warm-up call leaves the device's free memory and torch's
    allocated bytes unchanged (nothing is allocated on this path);
  * an A with more rows than the fixed scratch allows is refused with
    OCEAN_ERR_INVALID.
This file is collected last on purpose (name order)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
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


@pytest.mark.parametrize("bits", [32, 64])
def test_noalloc_matches_regular_entry_point_twice(bits):
    # first a skewed R-MAT (every class, bitmap rows included), then a smaller
    # uniform matrix: the second call reuses the scratch the first one filled
    cases = [M.rmat(17, 16, seed=31), M.uniform_random(40000, 12, seed=32)]
    g = SpGEMM()
    for A in cases:
        if bits == 64:
            A = A.widened()
        dA = DeviceCSR.from_host(A)
        got = noalloc_counts(dA, dA)
        want = g.symbolic(dA, dA).cpu().numpy().view(np.uint32)
        assert got.shape == want.shape
        assert np.array_equal(got, want)
        assert np.array_equal(got, O.symbolic(A, A).astype(np.uint32))


def test_noalloc_call_allocates_nothing():
    import torch
    A = M.rmat(16, 16, seed=34)
    dA = DeviceCSR.from_host(A)
    out = torch.empty(A.rows, dtype=torch.int32, device="cuda")
    av = dA.view()
    assert lib().ocean_symbolic_noalloc(ctypes.byref(av), ctypes.byref(av), out.data_ptr(), None) == 0  # warm-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    assert lib().ocean_symbolic_noalloc(ctypes.byref(av), ctypes.byref(av), out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_rejects_more_rows_than_scratch():
    A = M.uniform_random(MAX_ROWS + 1, 1, seed=33)
    dA = DeviceCSR.from_host(A)
    import torch
    out = torch.empty(A.rows, dtype=torch.int32, device="cuda")
    av = dA.view()
    rc = lib().ocean_symbolic_noalloc(ctypes.byref(av), ctypes.byref(av), out.data_ptr(), None)
    assert rc == 4
    assert b"more than the fixed scratch allows" in lib().ocean_last_error()
