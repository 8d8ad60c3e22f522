"""Windowed exact numeric kernel of the bitmap class (k_num_window): rows whose
output needs several shared-memory value windows (more than 12288 entries, or
a column span wider than 512K columns), rows with more than one chunk (1024)
of A entries (resume cursors in device memory), rows with saved bitmaps and
rows marked in the kernel, rows wider than 2^20 columns beside them (those run
in k_num_bitmap), 32- and 64-bit row pointers. Structure must match the CPU
oracle bit for bit, values within 1e-12 * sum |a*b|, and the output equals the
single-pass rank kernel's (numeric_windows off) in structure."""
import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import DeviceCSR, SpGEMM

pytestmark = pytest.mark.gpu

TOL = 1e-12


def heavy_mix(b_rows=40000, cols=1 << 20, cluster=4096, narrow_rows=0, seed=0):
    """A (2000 + narrow_rows rows) times B (b_rows x cols). B has power-law row
    lengths (up to 30000), every third row's columns in a cluster of `cluster`
    columns, the others uniform over all columns. Row 0 of A has 3000 entries,
    rows 1-40 have 100-900, the others 1-59, referencing mostly the long B
    rows; the extra `narrow_rows` rows each reference B rows 0 and 3 only."""
    rng = np.random.default_rng(seed)
    L = np.minimum(30000, (4 + 3000.0 / (np.arange(b_rows) + 1) ** 0.7 * 10).astype(np.int64))
    r = np.repeat(np.arange(b_rows), L)
    clustered = (np.arange(b_rows) % 3 == 0)[r]
    c = np.where(clustered, (r * 7919 + rng.integers(0, cluster, r.size)) % cols, rng.integers(0, cols, r.size))
    B = M.from_coo(b_rows, cols, r, c, rng.uniform(-1, 1, r.size))
    n_a = 2000
    anz = np.concatenate([[3000], rng.integers(100, 900, 40), rng.integers(1, 60, n_a - 41)])
    ar = np.repeat(np.arange(n_a), anz)
    ac = np.minimum((b_rows * rng.random(ar.size) ** 3).astype(np.int64), b_rows - 1)
    if narrow_rows:
        ar = np.concatenate([ar, np.repeat(np.arange(n_a, n_a + narrow_rows), 2)])
        ac = np.concatenate([ac, np.tile([0, 3], narrow_rows)])
        n_a += narrow_rows
    A = M.from_coo(n_a, b_rows, ar, ac, rng.uniform(-1, 1, ar.size))
    return A, B


def run(A, B, config):
    g = SpGEMM(config)
    dA = DeviceCSR.from_host(A)
    dB = DeviceCSR.from_host(B)
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


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("cache", [0.0, 0.25])
def test_windowed_rows_match_oracle(cache, bits):
    A, B = heavy_mix()
    if bits == 64:
        A, B = A.widened(), B.widened()
    # small_problem_nnz 0: read the class sizes back after the analysis, which
    # lets the symbolic pass save bitmaps (cache > 0) for the numeric pass
    C, st = run(A, B, {"bitmap_cache_fraction": cache, "small_problem_nnz": 0, "numeric_windows": True})
    check(A, B, C)
    assert st["decision"]["numeric_bitmap_kernel"] == "window"
    assert st["classes"]["numeric"]["bitmap"]["rows"] > 1000
    assert (st["decision"]["bitmap_cache_used_bytes"] > 0) == (cache > 0)


def test_windowed_equals_rank_kernel():
    A, B = heavy_mix(seed=3)
    Cw, stw = run(A, B, {"numeric_windows": True})
    Cr, str_ = run(A, B, {"numeric_windows": False})
    assert stw["decision"]["numeric_bitmap_kernel"] == "window"
    assert str_["decision"]["numeric_bitmap_kernel"] == "rank"
    assert np.array_equal(Cw.rowptr, Cr.rowptr) and np.array_equal(Cw.col, Cr.col)
    scale = np.maximum(np.abs(Cw.val), np.abs(Cr.val))
    assert np.all(np.abs(Cw.val - Cr.val) <= 1e-12 * np.maximum(scale, 1e-300) * 64)
    check(A, B, Cw)


def test_rows_wider_than_one_bitmap_beside_windowed_rows():
    # columns over 3 * 2^20: most bitmap-class rows are wider than 2^20 columns
    # (k_num_bitmap), the 300 extra rows span < 2^20 (k_num_window)
    A, B = heavy_mix(b_rows=20000, cols=3 << 20, cluster=1 << 18, narrow_rows=300, seed=5)
    p, lo, hi = O.row_stats(A, B)
    n = O.symbolic(A, B)
    span = hi.astype(np.int64) - lo.astype(np.int64) + 1
    assert ((n > 4096) & (span > 1 << 20)).sum() > 100
    assert ((n > 4096) & (span <= 1 << 20)).sum() >= 300
    C, st = run(A, B, {"numeric_windows": True})
    check(A, B, C)
    assert st["decision"]["numeric_bitmap_kernel"] == "window"


def test_dense_rows_many_windows_by_count():
    # 2048 rows of 64 random B rows of 400 entries over 2^16 columns: about
    # 21K outputs per row (a third of the span set), two windows by count
    rng = np.random.default_rng(8)
    A = M.from_coo(2048, 1 << 16, np.repeat(np.arange(2048), 64), rng.integers(0, 1 << 16, 2048 * 64),
                   rng.uniform(-1, 1, 2048 * 64))
    B = M.uniform_random(1 << 16, 400, seed=9)
    C, st = run(A, B, {"numeric_windows": True})
    check(A, B, C)
    assert st["classes"]["numeric"]["bitmap"]["rows"] == 2048
