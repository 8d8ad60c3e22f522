"""Host-buffer multiplies (ocean_spgemm_host) whose numeric phase runs in row
chunks of equal products, each chunk's C copied to the host while the next
ones compute: the result must equal the oracle's C and the unchunked result,
for 32- and 64-bit row pointers, several chunk counts, and inputs whose
product mass sits in a few rows (chunks that hold no row)."""
import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import SpGEMM

pytestmark = pytest.mark.gpu

# small inputs take the chunked path only with the product threshold at 0, the
# analysis read-back forced (it is skipped below 1 M entries of A) and the
# precise workflow (the only one that pipelines)
PIPE = {"host_pipeline_min_products": 0, "small_problem_nnz": 0, "force_workflow": 0}


def host_multiply(A, B, cfg):
    g = SpGEMM(cfg)
    C = g.multiply(A, B)
    st = g.get_stats()
    g.close()
    return C, st


def check(A, B, C):
    cp, cj, cx, ca = O.spgemm(A, B, with_abs=True)
    assert int(C.rowptr[-1]) == C.nnz == int(cp[-1])
    O.compare(C.rowptr, C.col, C.val, cp, cj, cx, ca, 1e-12)


def heavy_rows():
    """Uniform rows plus three rows that carry most of the products."""
    A = M.uniform_random(1 << 14, 8, seed=3)
    rows, cols, vals = [], [], []
    rng = np.random.default_rng(5)
    for r in range(A.rows):
        a, b = int(A.rowptr[r]), int(A.rowptr[r + 1])
        c = A.col[a:b]
        if r in (7, 4000, 9000):
            c = np.unique(np.concatenate([c, rng.choice(A.cols, 12000, replace=False)]))
        rows.append(np.full(c.size, r))
        cols.append(c)
        vals.append(rng.uniform(-1, 1, c.size))
    return M.from_coo(A.rows, A.cols, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


@pytest.mark.parametrize("chunks", [2, 8, 16])
def test_chunked_host_multiply_rmat(chunks):
    A = M.rmat(14, 16, seed=2)
    C, st = host_multiply(A, A, dict(PIPE, host_pipeline_chunks=chunks))
    assert st["decision"]["host_pipeline_chunks"] == chunks
    check(A, A, C)


def test_chunked_equals_unchunked_64bit_rowptr():
    A = M.rmat(13, 16, seed=9)
    cfg = dict(PIPE, output_rowptr_bits=64)
    C1, st1 = host_multiply(A, A, dict(cfg, host_pipeline_chunks=8))
    C0, st0 = host_multiply(A, A, dict(cfg, host_pipeline_chunks=0))
    assert st1["decision"]["host_pipeline_chunks"] == 8 and st0["decision"]["host_pipeline_chunks"] == 0
    assert C1.rowptr.dtype == np.uint64
    assert np.array_equal(C1.rowptr, C0.rowptr) and np.array_equal(C1.col, C0.col)
    # the bitmap and hash classes sum with atomics: two runs agree to rounding
    assert np.allclose(C1.val, C0.val, rtol=1e-12, atol=1e-12)
    check(A, A, C1)


def test_chunked_heavy_rows_and_empty_chunks():
    A = heavy_rows()
    C, st = host_multiply(A, A, dict(PIPE, host_pipeline_chunks=16))
    assert st["decision"]["host_pipeline_chunks"] == 16
    check(A, A, C)


def test_chunked_rectangular():
    A = M.rect_poisson(4096, 1 << 15, 12.0, seed=1)
    B = M.transpose(A)
    C, st = host_multiply(A, B, dict(PIPE, host_pipeline_chunks=4))
    assert st["decision"]["host_pipeline_chunks"] == 4
    check(A, B, C)


def test_small_host_multiply_is_not_chunked():
    A = M.laplacian_2d(64, 64, seed=0)
    C, st = host_multiply(A, A, {})
    assert st["decision"]["host_pipeline_chunks"] == 0
    check(A, A, C)
