"""Seeded synthetic CSR matrices and the reference's binary ``.hicsr`` format.

Generators stand in for the SuiteSparse matrices the reference evaluates on
(not available offline); they produce the shapes, sizes and value
distributions of the benchmark configurations:

* :func:`laplacian_2d` — 5-point Laplacian pattern on an nx×ny grid;
* :func:`rmat` — R-MAT power-law square matrix, duplicates merged;
* :func:`rect_poisson` — rectangular, Poisson(λ) entries per row, uniform columns;
* :func:`banded`, :func:`uniform_random`, :func:`block_diagonal` — the mixed
  families of the learned-estimator and batched workloads.

:func:`read_mtx` reads MatrixMarket coordinate files like the reference's
converter (utils/convert.cpp:83-240), so real matrices can be used where they
are available.

``.hicsr`` layout (reference src/CSR.cpp:70-152): an 80-byte header (9-byte
magic ``'H','i',1,'C','o','m','p','s','d'`` padded to 16, then eight uint64:
typesize, compresseddir, indexsize, fixedoffset, offsetsize, rows, cols, nnz),
a 16-byte state (double scaling, bool transpose, padding), then
``double data[nnz]``, ``uint32 col[nnz]``, ``uint32 rowptr[rows+1]``.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

from .ocean import HostCSR

HICSR_MAGIC = bytes([ord("H"), ord("i"), 1, ord("C"), ord("o"), ord("m"), ord("p"), ord("s"), ord("d")])


def _from_coo_sorted(rows: int, cols: int, r: np.ndarray, c: np.ndarray, v: np.ndarray) -> HostCSR:
    counts = np.bincount(r, minlength=rows).astype(np.uint64)
    rowptr = np.zeros(rows + 1, dtype=np.uint64)
    np.cumsum(counts, out=rowptr[1:])
    bits64 = rowptr[-1] >= 2**32
    return HostCSR(rows, cols, rowptr if bits64 else rowptr.astype(np.uint32),
                   c.astype(np.uint32), v.astype(np.float64))


def from_coo(rows: int, cols: int, r, c, v, sum_duplicates: bool = True) -> HostCSR:
    """CSR from COO triplets; duplicates are summed, columns sorted per row."""
    r = np.asarray(r, dtype=np.int64)
    c = np.asarray(c, dtype=np.int64)
    v = np.asarray(v, dtype=np.float64)
    key = r * max(cols, 1) + c
    order = np.argsort(key, kind="stable")
    key, v = key[order], v[order]
    if sum_duplicates and key.size:
        uniq, start = np.unique(key, return_index=True)
        v = np.add.reduceat(v, start)
        key = uniq
    return _from_coo_sorted(rows, cols, key // max(cols, 1), key % max(cols, 1), v)


def laplacian_2d(nx: int = 256, ny: int = 256, seed: int = 0) -> HostCSR:
    """5-point stencil pattern on an nx×ny grid, values uniform in [-1, 1]."""
    n = nx * ny
    idx = np.arange(n, dtype=np.int64)
    x, y = idx % nx, idx // nx
    rs, cs = [idx], [idx]
    for dx, dy in ((-1, 0), (1, 0), (0, -1), (0, 1)):
        ok = (x + dx >= 0) & (x + dx < nx) & (y + dy >= 0) & (y + dy < ny)
        rs.append(idx[ok])
        cs.append(idx[ok] + dx + dy * nx)
    r = np.concatenate(rs)
    c = np.concatenate(cs)
    key = np.sort(r * n + c)
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1.0, 1.0, key.size)
    return _from_coo_sorted(n, n, key // n, key % n, v)


def rmat(scale: int = 20, edge_factor: int = 16, probs=(0.57, 0.19, 0.19, 0.05), seed: int = 0,
         values: str = "uniform") -> HostCSR:
    """R-MAT: edge_factor·2^scale edges drawn by recursive quadrant choice with
    probabilities (a, b, c, d); duplicate edges merged; values U[-1,1]."""
    n = 1 << scale
    m = edge_factor * n
    rng = np.random.default_rng(seed)
    a, b, c, _ = probs
    r = np.zeros(m, dtype=np.int64)
    cc = np.zeros(m, dtype=np.int64)
    t1, t2, t3 = a, a + b, a + b + c
    for level in range(scale):
        u = rng.random(m)
        bit = np.int64(1) << np.int64(scale - 1 - level)
        rb = u >= t2             # quadrants c, d set the row bit
        cb = ((u >= t1) & (u < t2)) | (u >= t3)  # quadrants b, d set the column bit
        r |= rb.astype(np.int64) * bit
        cc |= cb.astype(np.int64) * bit
    key = np.unique(r * n + cc)
    if values == "uniform":
        v = rng.uniform(-1.0, 1.0, key.size)
    else:
        v = rng.standard_normal(key.size)
    return _from_coo_sorted(n, n, key // n, key % n, v)


def rect_poisson(rows: int = 262144, cols: int = 1048576, lam: float = 12.0, seed: int = 0) -> HostCSR:
    """rows×cols, Poisson(lam) entries per row at uniform random columns
    (duplicates within a row merged), values N(0,1)."""
    rng = np.random.default_rng(seed)
    k = rng.poisson(lam, rows).astype(np.int64)
    r = np.repeat(np.arange(rows, dtype=np.int64), k)
    c = rng.integers(0, cols, r.size, dtype=np.int64)
    key = np.unique(r * cols + c)
    v = rng.standard_normal(key.size)
    return _from_coo_sorted(rows, cols, key // cols, key % cols, v)


def banded(n: int, bandwidth: int, nnz_per_row: int, seed: int = 0) -> HostCSR:
    """Square, entries at random offsets in [-bandwidth, bandwidth] around the diagonal."""
    rng = np.random.default_rng(seed)
    k = min(nnz_per_row, 2 * bandwidth + 1)
    r = np.repeat(np.arange(n, dtype=np.int64), k)
    off = rng.integers(-bandwidth, bandwidth + 1, r.size)
    c = np.clip(r + off, 0, n - 1)
    key = np.unique(r * n + c)
    v = rng.uniform(-1.0, 1.0, key.size)
    return _from_coo_sorted(n, n, key // n, key % n, v)


def uniform_random(n: int, nnz_per_row: int, seed: int = 0) -> HostCSR:
    """Square, nnz_per_row uniform random columns per row (duplicates merged)."""
    rng = np.random.default_rng(seed)
    r = np.repeat(np.arange(n, dtype=np.int64), nnz_per_row)
    c = rng.integers(0, n, r.size, dtype=np.int64)
    key = np.unique(r * n + c)
    v = rng.uniform(-1.0, 1.0, key.size)
    return _from_coo_sorted(n, n, key // n, key % n, v)


def block_diagonal(n: int, block: int, nnz_per_row: int, seed: int = 0) -> HostCSR:
    """Square, each row's entries uniform inside its diagonal block of width `block`."""
    rng = np.random.default_rng(seed)
    k = min(nnz_per_row, block)
    r = np.repeat(np.arange(n, dtype=np.int64), k)
    start = (r // block) * block
    width = np.minimum(block, n - start)
    c = start + rng.integers(0, np.iinfo(np.int64).max, r.size) % width
    key = np.unique(r * n + c)
    v = rng.uniform(-1.0, 1.0, key.size)
    return _from_coo_sorted(n, n, key // n, key % n, v)


def transpose(m: HostCSR) -> HostCSR:
    """Explicit CSR transpose (used for A·Aᵀ)."""
    rp = m.rowptr.astype(np.int64)
    r = np.repeat(np.arange(m.rows, dtype=np.int64), np.diff(rp))
    c = m.col.astype(np.int64)
    order = np.lexsort((r, c))
    return _from_coo_sorted(m.cols, m.rows, c[order], r[order], m.val[order])


def write_hicsr(m: HostCSR, path) -> None:
    """Writes the reference's binary CSR format (src/CSR.cpp:70-152)."""
    if m.rowptr_bits == 64:
        raise ValueError(".hicsr stores 32-bit row offsets")
    hdr = HICSR_MAGIC + b"\0" * 7 + struct.pack("<8Q", 8, 0, 4, 0, 4, m.rows, m.cols, m.nnz)
    state = struct.pack("<d?7x", 1.0, False)
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(state)
        f.write(np.ascontiguousarray(m.val, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(m.col, dtype=np.uint32).tobytes())
        f.write(np.ascontiguousarray(m.rowptr, dtype=np.uint32).tobytes())


def read_hicsr(path) -> HostCSR:
    """Reads the reference's binary CSR format; raises ValueError on a bad file
    (reference: loadCSR throws, src/CSR.cpp:119-152)."""
    data = Path(path).read_bytes()
    if len(data) < 96:
        raise ValueError("Could not read CSR header")
    if data[:9] != HICSR_MAGIC:
        raise ValueError("File does not appear to be a CSR Matrix")
    typesize, _cd, _is, _fo, _os, rows, cols, nnz = struct.unpack_from("<8Q", data, 16)
    if typesize != 8:
        raise ValueError("File does not contain a CSR matrix with matching type")
    off = 96
    need = off + nnz * 8 + nnz * 4 + (rows + 1) * 4
    if len(data) < need:
        raise ValueError("Could not read CSR matrix data")
    val = np.frombuffer(data, np.float64, nnz, off).copy()
    off += nnz * 8
    col = np.frombuffer(data, np.uint32, nnz, off).copy()
    off += nnz * 4
    rowptr = np.frombuffer(data, np.uint32, rows + 1, off).copy()
    return HostCSR(int(rows), int(cols), rowptr, col, val)


def read_mtx(path) -> HostCSR:
    """Reads a MatrixMarket coordinate file the way the reference's converter
    does (utils/convert.cpp:83-240): header ``%%MatrixMarket matrix coordinate
    <type> <symmetry>``; type real, integer or double (values read as FP64),
    pattern (every value 1.0) or complex (the real part); symmetry general,
    symmetric or Hermitian, where every off-diagonal entry (r, c) is mirrored
    to (c, r) with the same value; 1-based indices checked against the size
    line; entries sorted by (row, column) with duplicates kept (in file order,
    where the reference's sort leaves their order open). Raises ValueError."""
    import io
    text = Path(path).read_text()
    lines = text.splitlines()
    if not lines or not lines[0].startswith("%%MatrixMarket matrix coordinate"):
        raise ValueError("Can only read MatrixMarket format that is in coordinate form")
    tok = lines[0].split()
    if len(tok) < 5:
        raise ValueError("incomplete MatrixMarket header")
    kind, sym = tok[3], tok[4]
    if kind not in ("pattern", "complex", "real", "integer", "double"):
        raise ValueError("MatrixMarket data type does not match matrix format")
    if sym not in ("general", "symmetric", "Hermitian"):
        raise ValueError("Can only read MatrixMarket format that is either symmetric, general or hermitian")
    i = 1
    while i < len(lines) and (not lines[i].strip() or lines[i].lstrip().startswith("%")):
        i += 1
    if i >= len(lines):
        raise ValueError("Failed to read matrix market header")
    size = lines[i].split()
    try:
        rows, cols, nnz = int(size[0]), int(size[1]), int(size[2])
    except (IndexError, ValueError):
        raise ValueError("Failed to read matrix market header")
    body = [ln for ln in lines[i + 1:] if ln.strip() and not ln.lstrip().startswith("%")]
    ncol = 2 if kind == "pattern" else 3
    if body:
        try:
            arr = np.loadtxt(io.StringIO("\n".join(body)), ndmin=2, usecols=range(ncol), dtype=np.float64)
        except ValueError as e:
            raise ValueError(f"Failed to read data from matrix market file: {e}")
    else:
        arr = np.zeros((0, ncol))
    r = arr[:, 0].astype(np.int64)
    c = arr[:, 1].astype(np.int64)
    v = np.ones(r.size) if kind == "pattern" else arr[:, 2].astype(np.float64)
    if r.size and (r.min() < 1 or r.max() > rows):
        raise ValueError("Row index out of bounds in matrix market file")
    if c.size and (c.min() < 1 or c.max() > cols):
        raise ValueError("Column index out of bounds in matrix market file")
    r, c = r - 1, c - 1
    if sym != "general":
        off = r != c
        # mirrored entry right after its original, as the reference appends it
        order = np.argsort(np.concatenate([np.arange(r.size) * 2, np.nonzero(off)[0] * 2 + 1]), kind="stable")
        r = np.concatenate([r, c[off]])[order]
        c2 = np.concatenate([c, arr[:, 0].astype(np.int64)[off] - 1])[order]
        v = np.concatenate([v, v[off]])[order]
        c = c2
    key = r * max(cols, 1) + c
    order = np.argsort(key, kind="stable")
    return _from_coo_sorted(rows, cols, r[order], c[order], v[order])

