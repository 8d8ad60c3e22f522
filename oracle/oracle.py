"""CPU oracle for the SpGEMM path — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference
legs may import this module, and only as the checker or the reported CPU
baseline. The product path (libocean.so) never calls it.

Wraps ``liboracle.so`` (built from ``oracle/gustavson.c`` by ``oracle/Makefile``):
a project-written FP64 Gustavson restating the reference's output semantics
(the reference has no CPU SpGEMM; see the header of gustavson.c for the
file:line anchors), plus MurmurHash3 and HyperLogLog restatements of
kernels/MurmurHash.cuh:44-98 and kernels/HLL.cuh:11-236. A pure-Python
Gustavson (:func:`py_spgemm`) restates the same rules once more for tiny
hand-checked cases.

Parity pins: MurmurHash3 against known answers produced by the reference's own
MurmurHash.cuh compiled on the host (``tests/golden/murmur3_kat.json``, made by
``tests/golden/make_golden.py``); the Gustavson against hand-computed products
(``tests/golden/tiny_cases.json``) and against scipy's sparse product on the
pattern and values. The reference has no CPU SpGEMM and no golden vectors of
its own, so the SpGEMM structure is pinned by hand-computed cases rather than
by reference outputs.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_lib = None


def build(force: bool = False) -> Path:
    """Builds liboracle.so with the committed Makefile (gcc + OpenMP)."""
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < (HERE / "gustavson.c").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return LIB_PATH


def _L():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
        L.oracle_row_stats.argtypes = [u64, u64, vp, vp, u64, u64, vp, vp, vp, vp, vp, i32]
        L.oracle_symbolic.argtypes = [u64, u64, vp, vp, u64, u64, vp, vp, u64, u64, u64, vp, i32]
        L.oracle_numeric.argtypes = [u64, u64, vp, vp, vp, u64, u64, vp, vp, vp, u64, u64, u64, vp, vp, vp, vp, i32]
        L.oracle_murmur3_u32.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_murmur3_u32.restype = ctypes.c_uint32
        L.oracle_murmur3_batch.argtypes = [vp, vp, u64, ctypes.c_uint32]
        L.oracle_murmur3_batch.restype = None
        L.oracle_hll_sketch_rows.argtypes = [u64, u64, vp, vp, i32, ctypes.c_uint32, vp]
        L.oracle_hll_sketch_rows.restype = None
        L.oracle_hll_estimate_union.argtypes = [vp, i32, vp, u64]
        L.oracle_hll_estimate_union.restype = ctypes.c_int64
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


def default_threads() -> int:
    return int(os.environ.get("OCEAN_ORACLE_THREADS", os.cpu_count() or 1))


def _wide(m):
    return np.ascontiguousarray(m.rowptr, dtype=np.uint64)


def row_stats(A, B, threads: int | None = None):
    """(products per row u64, lo u32, hi u32) — analysisKernel's per-row outputs."""
    prod = np.empty(A.rows, np.uint64)
    lo = np.empty(A.rows, np.uint32)
    hi = np.empty(A.rows, np.uint32)
    ap, bp = _wide(A), _wide(B)
    _L().oracle_row_stats(A.rows, A.nnz, _p(ap), _p(A.col), B.rows, B.nnz, _p(bp), _p(B.col),
                          _p(prod), _p(lo), _p(hi), threads or default_threads())
    return prod, lo, hi


def symbolic(A, B, r0: int = 0, r1: int | None = None, threads: int | None = None) -> np.ndarray:
    """Exact output count per row for rows [r0, r1)."""
    r1 = A.rows if r1 is None else r1
    out = np.empty(r1 - r0, np.uint64)
    ap, bp = _wide(A), _wide(B)
    rc = _L().oracle_symbolic(A.rows, A.nnz, _p(ap), _p(A.col), B.rows, B.nnz, _p(bp), _p(B.col), B.cols,
                              r0, r1, _p(out), threads or default_threads())
    if rc:
        raise MemoryError("oracle_symbolic failed")
    return out


def spgemm(A, B, r0: int = 0, r1: int | None = None, with_abs: bool = False, threads: int | None = None):
    """C rows [r0, r1) of A·B: returns (rowptr u64 relative to row r0, col, val[, abs])."""
    r1 = A.rows if r1 is None else r1
    t = threads or default_threads()
    counts = symbolic(A, B, r0, r1, t)
    cp = np.zeros(r1 - r0 + 1, np.uint64)
    np.cumsum(counts, out=cp[1:])
    nnz = int(cp[-1])
    cj = np.empty(nnz, np.uint32)
    cx = np.empty(nnz, np.float64)
    ca = np.empty(nnz, np.float64) if with_abs else None
    ap, bp = _wide(A), _wide(B)
    rc = _L().oracle_numeric(A.rows, A.nnz, _p(ap), _p(A.col), _p(A.val), B.rows, B.nnz, _p(bp), _p(B.col),
                             _p(B.val), B.cols, r0, r1, _p(cp), _p(cj), _p(cx), _p(ca) if ca is not None else 0, t)
    if rc:
        raise RuntimeError(f"oracle_numeric failed ({rc})")
    return (cp, cj, cx, ca) if with_abs else (cp, cj, cx)


def murmur3(keys: np.ndarray, seed: int = 1234) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    out = np.empty_like(keys)
    _L().oracle_murmur3_batch(_p(keys), _p(out), keys.size, seed)
    return out


def hll_sketch_rows(B, log2p: int, seed: int = 1234) -> np.ndarray:
    out = np.empty(B.rows * (1 << log2p), np.uint8)
    bp = _wide(B)
    _L().oracle_hll_sketch_rows(B.rows, B.nnz, _p(bp), _p(B.col), log2p, seed, _p(out))
    return out


def hll_estimate_union(sketches: np.ndarray, log2p: int, rows: np.ndarray) -> int:
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    return int(_L().oracle_hll_estimate_union(_p(sketches), log2p, _p(rows), rows.size))


# ----------------------------------------------------------------- pure Python
def py_murmur3(key: int, seed: int = 1234) -> int:
    """Pure-Python MurmurHash3_x86_32 of one 4-byte little-endian key."""
    M = 0xFFFFFFFF
    k = (key * 0xCC9E2D51) & M
    k = ((k << 15) | (k >> 17)) & M
    k = (k * 0x1B873593) & M
    h = seed ^ k
    h = ((h << 13) | (h >> 19)) & M
    h = (h * 5 + 0xE6546B64) & M
    h ^= 4
    h ^= h >> 16
    h = (h * 0x85EBCA6B) & M
    h ^= h >> 13
    h = (h * 0xC2B2AE35) & M
    h ^= h >> 16
    return h


def py_spgemm(A, B):
    """Tiny pure-Python Gustavson with the same rules (structural zeros kept,
    columns ascending, last row ends at nnz). Returns (rowptr, col, val)."""
    def rng(m, r):
        return int(m.rowptr[r]), (m.nnz if r + 1 == m.rows else int(m.rowptr[r + 1]))

    rp, cj, cx = [0], [], []
    for i in range(A.rows):
        acc = {}
        a0, a1 = rng(A, i)
        for k in range(a0, a1):
            j = int(A.col[k])
            b0, b1 = rng(B, j)
            for q in range(b0, b1):
                c = int(B.col[q])
                acc[c] = acc.get(c, 0.0) + float(A.val[k]) * float(B.val[q])
        for c in sorted(acc):
            cj.append(c)
            cx.append(acc[c])
        rp.append(len(cj))
    return np.array(rp, np.uint64), np.array(cj, np.uint32), np.array(cx, np.float64)


def compare(rowptr, col, val, ref_rowptr, ref_col, ref_val, ref_abs=None, tol: float = 1e-12):
    """Structure must match exactly; each value must satisfy
    |x - y| <= tol * sum_k |a_ik b_kj| (or tol * max(|x|,|y|) without abs)."""
    rowptr = np.asarray(rowptr, np.uint64)
    ref_rowptr = np.asarray(ref_rowptr, np.uint64)
    if rowptr.shape != ref_rowptr.shape or not np.array_equal(rowptr - rowptr[0], ref_rowptr - ref_rowptr[0]):
        bad = np.nonzero((rowptr - rowptr[0]) != (ref_rowptr - ref_rowptr[0]))[0] if rowptr.shape == ref_rowptr.shape else []
        raise AssertionError(f"row pointers differ (first rows {list(bad[:5])})")
    if not np.array_equal(np.asarray(col, np.uint32), np.asarray(ref_col, np.uint32)):
        bad = np.nonzero(np.asarray(col) != np.asarray(ref_col))[0]
        raise AssertionError(f"column ids differ at {bad.size} entries (first {list(bad[:5])})")
    val = np.asarray(val, np.float64)
    ref_val = np.asarray(ref_val, np.float64)
    scale = np.asarray(ref_abs, np.float64) if ref_abs is not None else np.maximum(np.abs(val), np.abs(ref_val))
    err = np.abs(val - ref_val)
    bad = err > tol * scale
    if bad.any():
        i = int(np.nonzero(bad)[0][0])
        raise AssertionError(f"{int(bad.sum())} values outside tolerance; first at {i}: {val[i]} vs {ref_val[i]}")
    rel = err / np.where(scale > 0, scale, 1.0)
    return float(rel.max()) if rel.size else 0.0
