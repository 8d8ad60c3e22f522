"""Direct-addressed hash classes: a row whose output column span fits its
class table (span <= slots) is accumulated at slot = column - lo, without
probing, and written by an ordered compaction instead of a sort. Structure
must match the oracle bit for bit, values within 1e-12 of sum |a_ik * b_kj|."""
import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M

from test_gpu_parity import NUM_BINS, SYM_BINS, check, multiply_device

pytestmark = pytest.mark.gpu

HASH = ["hash_s", "hash_m", "hash_l"]
NUM_SLOTS = {"hash_s": 1024, "hash_m": 4096, "hash_l": 8192}


def _rows_of(m):
    return np.repeat(np.arange(m.rows), np.diff(m.rowptr.astype(np.int64)[:m.rows + 1]))


@pytest.mark.parametrize("num", HASH)
@pytest.mark.parametrize("sym", HASH)
def test_narrow_rows_every_hash_class(sym, num):
    A = M.banded(8000, 33, 16, seed=7)  # spans <= 133 columns: every row is direct
    C, _ = multiply_device(A, A, {"force_sym_bin": SYM_BINS[sym], "force_num_bin": NUM_BINS[num]})
    check(A, A, C)


def test_direct_and_hashed_rows_in_one_launch():
    # narrow banded rows on top, wide uniform-random rows below, one class for all
    Nb = M.banded(4096, 20, 12, seed=1)
    U = M.uniform_random(4096, 12, seed=2)
    r = np.concatenate([_rows_of(Nb), 4096 + _rows_of(U)])
    c = np.concatenate([Nb.col, U.col]).astype(np.int64)
    v = np.concatenate([Nb.val, U.val])
    A = M.from_coo(8192, 4096, r, c, v)
    R = M.uniform_random(4096, 6, seed=3)
    rb = _rows_of(R)
    B = M.from_coo(4096, 4096, rb, (rb + R.col.astype(np.int64) % 7) % 4096, R.val)  # 6 nearby columns per row
    for sym, num in (("hash_s", "hash_s"), ("hash_m", "hash_l")):
        C, _ = multiply_device(A, B, {"force_sym_bin": SYM_BINS[sym], "force_num_bin": NUM_BINS[num]})
        check(A, B, C)


@pytest.mark.parametrize("num", HASH)
def test_span_at_the_slot_count(num):
    # row 0 spans exactly the slot count (direct), row 1 one column more
    # (hashed); both reach column 5 twice
    T = NUM_SLOTS[num]
    B = M.from_coo(5, 2 * T + 8, np.array([0, 1, 2, 3, 4, 4]), np.array([0, T - 1, T, 5, 5, T - 1]),
                   np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0]))
    A = M.from_coo(2, 5, np.array([0, 0, 0, 0, 1, 1, 1]), np.array([0, 1, 3, 4, 0, 2, 3]),
                   np.array([1.5, -2.0, 0.5, 1.0, 3.0, -1.0, 2.0]))
    for sym in HASH:
        C, _ = multiply_device(A, B, {"force_sym_bin": SYM_BINS[sym], "force_num_bin": NUM_BINS[num]})
        check(A, B, C)
        assert list(C.col[:int(C.rowptr[1])]) == [0, 5, T - 1]
        assert list(C.col[int(C.rowptr[1]):int(C.rowptr[2])]) == [0, 5, T]


@pytest.mark.parametrize("wf", [1, 2])
def test_direct_rows_in_the_estimated_workflows(wf):
    # estimation (HLL-sized slots) and ultra-sparse (product-sized slots) write
    # through the count / overflow path of the same kernels
    A = M.block_diagonal(16384, 128, 24, seed=9)
    C, st = multiply_device(A, A, {"force_workflow": wf, "force_num_bin": NUM_BINS["hash_s"]})
    check(A, A, C)
    assert st["decision"]["workflow"] == wf


def test_direct_rows_fill_every_slot():
    # 1024-column blocks forced into the 1024-slot class: up to 1024 entries a
    # row, twice the sort capacity of a hashed row, written in order
    R = M.block_diagonal(4096, 1024, 64, seed=2)
    C, _ = multiply_device(R, R, {"force_num_bin": NUM_BINS["hash_s"]})
    check(R, R, C)
    assert int(np.diff(C.rowptr.astype(np.int64)).max()) > 512


@pytest.mark.parametrize("prefer", [True, False])
def test_mid_rows_with_narrow_spans_take_a_direct_table(prefer):
    # 512-wide bands of 32 entries: ~1000 outputs a row over ~1000 columns.
    # With prefer_direct_hash (the default) the rows go to the 4096-slot class
    # and are addressed directly; without it they go to the bitmap class.
    A = M.banded(20000, 512, 32, seed=3)
    C, st = multiply_device(A, A, {"prefer_direct_hash": prefer})
    check(A, A, C)
    b2 = st["binning_2"]
    heavy = b2[NUM_BINS["hash_m"]] if prefer else b2[NUM_BINS["bitmap"]]
    assert heavy > 0.9 * A.rows
    assert st["host_timeline_ms"]["analysis"] <= st["host_timeline_ms"]["launched"]
