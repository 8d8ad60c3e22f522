"""CPU tests: the oracle against hand-computed products, scipy and the
reference's own MurmurHash3 known answers; generators; .hicsr I/O."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import HostCSR


def to_scipy(m):
    return sp.csr_matrix((m.val, m.col.astype(np.int64), m.rowptr.astype(np.int64)), shape=(m.rows, m.cols))


def test_oracle_tiny_cases(tiny_cases):
    for name, A, B, (rp, col, val) in tiny_cases:
        cp, cj, cx = O.spgemm(A, B)
        O.compare(cp, cj, cx, rp, col, val, tol=0.0)
        prp, pcj, pcx = O.py_spgemm(A, B)
        O.compare(prp, pcj, pcx, rp, col, val, tol=0.0)


def test_oracle_keeps_cancelled_entries(tiny_cases):
    name, A, B, (rp, col, val) = [c for c in tiny_cases if c[0] == "cancellation_to_zero"][0]
    cp, cj, cx = O.spgemm(A, B)
    assert cx[0] == 0.0 and cj[0] == 0 and cp[-1] == 2


@pytest.mark.parametrize("gen", ["uniform", "banded", "block", "rect", "rmat"])
def test_oracle_matches_scipy(gen):
    if gen == "uniform":
        A = M.uniform_random(3000, 9, seed=1); B = A
    elif gen == "banded":
        A = M.banded(4000, 20, 12, seed=2); B = A
    elif gen == "block":
        A = M.block_diagonal(4096, 64, 16, seed=3); B = A
    elif gen == "rect":
        A = M.rect_poisson(3000, 9000, 12.0, seed=4); B = M.transpose(A)
    else:
        A = M.rmat(12, 8, seed=5); B = A
    cp, cj, cx, ca = O.spgemm(A, B, with_abs=True)
    # structure: scipy on all-ones patterns keeps every touched column
    P = (abs(to_scipy(A)).astype(bool).astype(np.float64) @ abs(to_scipy(B)).astype(bool).astype(np.float64)).tocsr()
    P.sort_indices()
    assert np.array_equal(cp, P.indptr.astype(np.uint64))
    assert np.array_equal(cj, P.indices.astype(np.uint32))
    # values: scipy's product, entry by entry where scipy kept the entry
    S = (to_scipy(A) @ to_scipy(B)).tocsr()
    S.sort_indices()
    dense_ref = S.toarray() if A.rows * B.cols <= 4e7 else None
    if dense_ref is not None:
        rows = np.repeat(np.arange(A.rows), np.diff(cp.astype(np.int64)))
        ref = dense_ref[rows, cj.astype(np.int64)]
        assert np.all(np.abs(cx - ref) <= 1e-12 * np.maximum(ca, 1e-300))


def test_oracle_row_ranges_match_full():
    A = M.rmat(11, 8, seed=7)
    cp, cj, cx = O.spgemm(A, A)
    r0, r1 = 300, 1200
    p2, j2, x2 = O.spgemm(A, A, r0, r1)
    s, e = int(cp[r0]), int(cp[r1])
    assert np.array_equal(p2 + cp[r0], cp[r0:r1 + 1])
    assert np.array_equal(j2, cj[s:e]) and np.array_equal(x2, cx[s:e])


def test_row_stats():
    A = M.laplacian_2d(32, 32, 0)
    prod, lo, hi = O.row_stats(A, A)
    rp = A.rowptr.astype(np.int64)
    for i in (0, 17, 500, 1023):
        ks = A.col[rp[i]:rp[i + 1]]
        assert prod[i] == sum(int(rp[k + 1] - rp[k]) for k in ks)
        assert lo[i] == min(A.col[rp[k]] for k in ks) and hi[i] == max(A.col[rp[k + 1] - 1] for k in ks)


def test_murmur3_oracle_matches_reference_kat(murmur_kat):
    keys, hashes = murmur_kat
    assert np.array_equal(O.murmur3(keys, 1234), hashes)
    for k, h in list(zip(keys, hashes))[:64]:
        assert O.py_murmur3(int(k), 1234) == int(h)


def test_hll_sketch_rules():
    # idx = low log2p bits of the hash; value = clz(hash) + 1 capped at 32 - log2p + 1
    B = HostCSR(1, 1 << 20, np.array([0, 4000], np.uint32), np.arange(0, 4000 * 200, 200, dtype=np.uint32),
                np.ones(4000))
    for log2p in (5, 6):
        sk = O.hll_sketch_rows(B, log2p)
        h = O.murmur3(B.col)
        m = 1 << log2p
        ref = np.zeros(m, np.uint8)
        for x in h:
            x = int(x)
            v = min((32 - x.bit_length()) + 1, 32 - log2p + 1)
            ref[x & (m - 1)] = max(ref[x & (m - 1)], v)
        assert np.array_equal(sk, ref)
        est = O.hll_estimate_union(sk, log2p, np.array([0]))
        assert 0.5 * 4000 < est < 1.6 * 4000


def test_generators_match_known_sizes():
    """The Laplacian 256x256 workload has 326,656 entries, 1,629,192 products and
    846,852 output entries; the rect and R-MAT generators keep their densities."""
    A = M.laplacian_2d(256, 256, 0)
    assert (A.rows, A.nnz) == (65536, 326656)
    prod, _, _ = O.row_stats(A, A)
    assert int(prod.sum()) == 1629192 and int(prod.max()) == 25
    assert int(O.symbolic(A, A).sum()) == 846852
    R = M.rect_poisson(4096, 16384, 12.0, seed=0)
    assert abs(R.nnz / R.rows - 12.0) < 0.3
    G = M.rmat(14, 16, seed=0)
    assert np.all(np.diff(G.rowptr.astype(np.int64)) >= 0) and G.nnz < 16 << 14


def test_generators_are_seeded():
    a, b = M.rmat(10, 8, seed=3), M.rmat(10, 8, seed=3)
    assert np.array_equal(a.col, b.col) and np.array_equal(a.val, b.val)
    c = M.rmat(10, 8, seed=4)
    assert not (a.nnz == c.nnz and np.array_equal(a.col, c.col))


def test_columns_sorted_and_unique():
    for m in (M.rmat(10, 8, seed=1), M.banded(500, 5, 4, seed=1), M.block_diagonal(512, 32, 8, seed=1)):
        rp = m.rowptr.astype(np.int64)
        for i in range(m.rows):
            seg = m.col[rp[i]:rp[i + 1]]
            assert np.all(np.diff(seg.astype(np.int64)) > 0)


def test_hicsr_roundtrip(tmp_path):
    A = M.rmat(9, 6, seed=2)
    p = tmp_path / "a.mtxd_.hicsr"
    M.write_hicsr(A, p)
    raw = p.read_bytes()
    assert raw[:9] == M.HICSR_MAGIC and len(raw) == 96 + A.nnz * 12 + (A.rows + 1) * 4
    B = M.read_hicsr(p)
    assert (B.rows, B.cols, B.nnz) == (A.rows, A.cols, A.nnz)
    assert np.array_equal(B.rowptr, A.rowptr) and np.array_equal(B.col, A.col) and np.array_equal(B.val, A.val)


def test_hicsr_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.hicsr"
    p.write_bytes(b"not a csr file at all" * 10)
    with pytest.raises(ValueError, match="does not appear"):
        M.read_hicsr(p)
    p.write_bytes(b"\0" * 10)
    with pytest.raises(ValueError, match="header"):
        M.read_hicsr(p)


def test_compare_detects_mistakes():
    A = M.uniform_random(200, 6, seed=9)
    cp, cj, cx, ca = O.spgemm(A, A, with_abs=True)
    bad = cx.copy(); bad[5] += 1e-6 * max(1.0, ca[5])
    with pytest.raises(AssertionError):
        O.compare(cp, cj, bad, cp, cj, cx, ca)
    badc = cj.copy(); badc[3] += 1
    with pytest.raises(AssertionError):
        O.compare(cp, badc, cx, cp, cj, cx, ca)
