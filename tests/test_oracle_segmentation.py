"""CPU tests of the segmentation restatement: a hand-checked 16 x 16 case and
the class each designed matrix family must get (kernels/Segmentation.cuh of
the reference)."""
import numpy as np

from oracle import oracle as O
from oracle import segmentation as S
from research_b200 import matrices as M


def two_blocks():
    # dense 4 x 4 blocks at rows/cols 0-3 and 8-11 of a 16 x 16 matrix
    r, c = [], []
    for base in (0, 8):
        for i in range(4):
            for j in range(4):
                r.append(base + i)
                c.append(base + j)
    return M.from_coo(16, 16, np.array(r), np.array(c), np.ones(len(r)))


def test_hand_checked_two_blocks():
    A = two_blocks()
    g = S.segment(A, A, grid_max=8, hot_k=2.0, min_segment_rows=1)
    # 8 x 8 grid of 2 x 2 tiles; 8 tiles hold 4 entries each: mean 0.5,
    # stddev sqrt(2 - 0.25), threshold 3.15 -> exactly the block tiles are hot
    assert (g["grid_h"], g["grid_w"], g["tile_rows"], g["tile_cols"]) == (8, 8, 2, 2)
    assert g["density_mean"] == 0.5
    assert g["density_stddev"] == np.sqrt(1.75)
    # labels 0 (tiles 0, 1, 8, 9) and 36 (36, 37, 44, 45): two rounds change labels
    assert g["cc_iterations"] == 2
    assert g["num_components"] == 2
    segs = g["segments"]
    assert [(s["row_start"], s["row_end"]) for s in segs] == [(0, 4), (4, 8), (8, 12), (12, 16)]
    assert [s["class"] for s in segs] == ["DENSE", "SPARSE_UNIFORM", "DENSE", "SPARSE_UNIFORM"]
    s0 = segs[0]
    assert (s0["sum_products"], s0["sum_a_nnz"], s0["col_left"], s0["col_right"]) == (64, 16, 0, 3)
    assert (s0["mean_row_len"], s0["var_row_len"], s0["local_er"]) == (16.0, 0.0, 4.0)
    assert (s0["max_b_row_len"], s0["max_a_row_len"]) == (4, 4)
    s1 = segs[1]  # rows without products: span (0, 0), nothing else
    assert (s1["sum_products"], s1["col_left"], s1["col_right"], s1["mean_row_len"]) == (0, 0, 0, 0.0)
    assert segs[2]["col_left"] == 8 and segs[2]["col_right"] == 11


def test_short_bands_join_the_previous_one():
    A = two_blocks()
    g = S.segment(A, A, grid_max=8, hot_k=2.0, min_segment_rows=5)
    assert [(s["row_start"], s["row_end"]) for s in g["segments"]] == [(0, 16)]
    assert g["num_components"] == 1


def test_row_stats_match_the_gustavson_oracle():
    A = M.rmat(12, 8, seed=5)
    prod, lo, hi, anz, maxb = S.row_stats(A, A)
    p2, l2, h2 = O.row_stats(A, A)
    assert np.array_equal(prod, p2.astype(np.int64))
    assert np.array_equal(lo, l2.astype(np.int64))
    assert np.array_equal(hi, h2.astype(np.int64))
    assert np.array_equal(anz, np.diff(A.rowptr.astype(np.int64)))
    blen = np.diff(A.rowptr.astype(np.int64))
    for r in range(0, A.rows, 97):
        cols = A.col[A.rowptr[r]:A.rowptr[r + 1]].astype(np.int64)
        assert maxb[r] == (blen[cols].max() if cols.size else 0)


def classes(A, **kw):
    return [s["class"] for s in S.segment(A, A, **kw)["segments"]]


def test_classes_of_designed_families():
    # narrow diagonal band, 16 entries per row: every 4096-row band spans
    # ~1/256 of the columns with products / entries = 16 -> BANDED
    A = M.banded(1 << 20, 16, 16, seed=6)
    c = classes(A)
    assert len(c) == 256 and set(c) == {"BANDED"}
    # products per row fill far more than 25% of the span -> DENSE
    assert set(classes(M.uniform_random(2000, 200, seed=7))) == {"DENSE"}
    # uniform sparse rows -> SPARSE_UNIFORM
    assert set(classes(M.uniform_random(100000, 8, seed=8))) == {"SPARSE_UNIFORM"}
    # a skewed R-MAT: heavy-tailed products per row -> POWER_LAW
    assert "POWER_LAW" in classes(M.rmat(16, 8, seed=9))


def test_segments_partition_the_rows():
    for A in (M.rmat(14, 8, seed=10), M.block_diagonal(50000, 256, 8, seed=11), M.laplacian_2d(300, 200)):
        segs = S.segment(A, A)["segments"]
        assert segs[0]["row_start"] == 0 and segs[-1]["row_end"] == A.rows
        for a, b in zip(segs, segs[1:]):
            assert a["row_end"] == b["row_start"]
        assert sum(s["sum_products"] for s in segs) == int(S.row_stats(A, A)[0].sum())
