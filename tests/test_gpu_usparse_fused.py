"""Fused ultra-sparse multiply (k_usp_fused): one launch merges every row (at
most 256 products) in registers or shared memory, finds its tile's output
offset by a decoupled look-back and writes C in place. Checked against the CPU
oracle (structure bit for bit, values within 1e-12 * sum |a*b|) on the
Laplacian 256^2, the rectangular A*A^T (rows up to 131 products: the
shared-memory sort path), rows at every product-count boundary
(0, 1, 32, 33, 64, 65, 128, 129, 256), the last tile partly filled, forced
64-bit output row pointers, and inputs the fused path does not take (a row
over 256 products; fused_ultrasparse off), which must give the same C."""
import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import DeviceCSR, SpGEMM

pytestmark = pytest.mark.gpu

TOL = 1e-12


FUSED = {"fused_ultrasparse": True}


def run(A, B, config=None):
    g = SpGEMM({**FUSED, **(config or {})})
    dA = DeviceCSR.from_host(A)
    dB = dA if B is A else DeviceCSR.from_host(B)
    C = g.multiply(dA, dB)
    h = C.download()
    C.free()
    st = g.get_stats()
    g.close()
    return h, st


def check(A, B, C):
    cp, cj, cx, ca = O.spgemm(A, B, with_abs=True)
    assert int(C.rowptr[-1]) == C.nnz == int(cp[-1])
    return O.compare(C.rowptr, C.col, C.val, cp, cj, cx, ca, TOL)


def test_laplacian_fused():
    A = M.laplacian_2d(256, 256, seed=0)
    C, st = run(A, A)
    check(A, A, C)
    assert st["decision"]["fused_ultrasparse"] is True
    assert st["C"]["nnz"] == 846852


def test_rect_fused_with_smem_sorted_rows():
    A = M.rect_poisson(262144, 1048576, 12.0, seed=0)
    B = M.transpose(A)
    p, _, _ = O.row_stats(A, B)
    assert p.max() > 128  # some rows take the shared-memory sort
    C, st = run(A, B)
    check(A, B, C)
    assert st["decision"]["fused_ultrasparse"] is True


def boundary_matrix(seed=0):
    """Rows whose product counts sit on every path boundary: row i has A
    entries pointing at B rows whose lengths add up to a chosen count; B rows
    have random columns over 5000 (repeats merge)."""
    rng = np.random.default_rng(seed)
    targets = [0, 1, 2, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 200, 255, 256] * 3 + [5] * 11
    nb = 4000
    blen = rng.integers(1, 9, nb)
    brows = np.repeat(np.arange(nb), blen)
    bcols = rng.integers(0, 5000, brows.size)
    B = M.from_coo(nb, 5000, brows, bcols, rng.uniform(-1, 1, brows.size), sum_duplicates=False)
    blen = np.diff(B.rowptr.astype(np.int64))
    ar, ac = [], []
    for i, t in enumerate(targets):
        got = 0
        used = set()
        while got < t:
            need = t - got
            cand = np.nonzero((blen <= need) & (blen > 0))[0]
            j = int(rng.choice(cand))
            if j in used:
                continue
            used.add(j)
            ar.append(i)
            ac.append(j)
            got += int(blen[j])
    A = M.from_coo(len(targets), nb, np.array(ar, np.int64), np.array(ac, np.int64),
                   rng.uniform(-1, 1, len(ar)))
    return A, B, targets


def test_product_count_boundaries_and_partial_last_tile():
    A, B, targets = boundary_matrix()
    p, _, _ = O.row_stats(A, B)
    assert list(p.astype(int)) == targets
    for cfg in ({}, {"output_rowptr_bits": 64}):
        C, st = run(A, B, {"force_workflow": 2, **cfg})
        check(A, B, C)
        assert st["decision"]["fused_ultrasparse"] is True


def test_row_over_256_products_is_not_fused_and_matches():
    A = M.uniform_random(5000, 6, seed=4)
    rp = A.rowptr.astype(np.int64)
    # one dense row of A: 60 entries x about 6 per B row > 256 products
    r = np.concatenate([np.repeat(np.arange(A.rows), np.diff(rp)), np.zeros(60, np.int64)])
    c = np.concatenate([A.col.astype(np.int64), np.arange(60) * 7])
    A2 = M.from_coo(A.rows, A.cols, r, c, np.ones(r.size))
    C, st = run(A2, A2)
    check(A2, A2, C)
    assert st["decision"]["fused_ultrasparse"] is False


@pytest.mark.parametrize("gen", ["laplacian", "uniform"])
def test_fused_equals_unfused(gen):
    A = M.laplacian_2d(300, 200, seed=3) if gen == "laplacian" else M.uniform_random(50000, 7, seed=5)
    Cf, stf = run(A, A, {})
    assert sum(stf["binning_2"]) == int(np.count_nonzero(np.diff(Cf.rowptr.astype(np.int64))))
    Cu, stu = run(A, A, {"fused_ultrasparse": False})
    assert stf["decision"]["fused_ultrasparse"] is True and stu["decision"]["fused_ultrasparse"] is False
    assert np.array_equal(Cf.rowptr, Cu.rowptr) and np.array_equal(Cf.col, Cu.col)
    check(A, A, Cf)


def test_empty_and_repeated_calls():
    g = SpGEMM(FUSED)
    A = M.laplacian_2d(64, 64, seed=9)
    dA = DeviceCSR.from_host(A)
    for _ in range(3):
        C = g.multiply(dA, dA)
        h = C.download()
        C.free()
        check(A, A, h)
    E = M.from_coo(10, 10, np.array([], np.int64), np.array([], np.int64), np.array([]))
    C = g.multiply(E, E)
    assert C.nnz == 0 and list(C.rowptr) == [0] * 11
