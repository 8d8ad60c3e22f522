"""The .mtx -> .hicsr converter against the reference's own converter
(utils/convert.cpp, built from its source by `make -C oracle refconvert` into
oracle/_ref/convert_ref): both convert the same MatrixMarket files and the
outputs must agree byte for byte, except the header's padding bytes (the 7
bytes after the 9-byte magic and the 7 after the State flag), which the
reference writes from uninitialised stack memory. Where duplicate (row,
column) entries are kept, the reference's std::sort leaves their relative order
open, so duplicates are compared as sets of values per position group.
Cases: general real with comments and blank lines, integer, pattern,
symmetric, Hermitian complex (real part), duplicates, empty rows and trailing
empty rows, a larger random matrix."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from research_b200.convert import main as convert_main

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref" / "convert_ref"

PAD = set(range(9, 16)) | set(range(88, 96))  # header padding, State padding


def _need_ref():
    if not REF.exists():
        pytest.skip("reference converter not built (make -C oracle refconvert needs the reference source tree)")


def both(tmp_path, text):
    src = tmp_path / "in.mtx"
    src.write_text(text)
    ours, ref = tmp_path / "ours.hicsr", tmp_path / "ref.hicsr"
    assert convert_main([str(src), str(ours)]) == 0
    r = subprocess.run([str(REF), str(src), str(ref)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return ours.read_bytes(), ref.read_bytes()


def same_bytes(a: bytes, b: bytes):
    assert len(a) == len(b)
    diff = [i for i in range(min(len(a), 4096)) if a[i] != b[i] and i not in PAD]
    assert not diff, diff[:10]
    assert a[96:] == b[96:]


def split(blob: bytes):
    rows, cols, nnz = np.frombuffer(blob, np.uint64, 3, 16 + 5 * 8)
    off = 96
    val = np.frombuffer(blob, np.float64, int(nnz), off)
    off += 8 * int(nnz)
    col = np.frombuffer(blob, np.uint32, int(nnz), off)
    off += 4 * int(nnz)
    rp = np.frombuffer(blob, np.uint32, int(rows) + 1, off)
    return int(rows), int(cols), rp, col, val


CASES = {
    "general_real": """%%MatrixMarket matrix coordinate real general
% comment line
4 5 6

1 1 1.5
4 5 -2
1 3 0.25
% another comment
2 2 7
4 1 1e-3
3 3 -0.5
""",
    "integer": """%%MatrixMarket matrix coordinate integer general
3 3 4
3 3 9
1 2 -4
2 1 5
1 1 1
""",
    "pattern": """%%MatrixMarket matrix coordinate pattern general
3 4 4
3 4
1 2
2 1
1 4
""",
    "symmetric": """%%MatrixMarket matrix coordinate real symmetric
4 4 5
1 1 2.5
2 1 -1
3 2 0.75
4 4 3
4 1 0.125
""",
    "hermitian_complex": """%%MatrixMarket matrix coordinate complex Hermitian
3 3 4
1 1 2.0 0.0
2 1 1.5 -0.5
3 1 -2.25 1.0
3 3 4.0 0.0
""",
    "empty_rows": """%%MatrixMarket matrix coordinate real general
6 3 3
2 1 1
2 3 2
4 2 3
""",
}


@pytest.mark.parametrize("name", list(CASES))
def test_converter_bytes_match_reference(tmp_path, name):
    _need_ref()
    ours, ref = both(tmp_path, CASES[name])
    same_bytes(ours, ref)


def test_random_matrix_bytes_match_reference(tmp_path):
    _need_ref()
    rng = np.random.default_rng(3)
    n, m, k = 3000, 2000, 40000
    r = rng.integers(1, n + 1, k)
    c = rng.integers(1, m + 1, k)
    keep = np.unique(r * (m + 1) + c, return_index=True)[1]  # distinct positions: the order is fully fixed
    r, c = r[keep], c[keep]
    v = rng.normal(0, 1, r.size)
    lines = [f"%%MatrixMarket matrix coordinate real general", f"{n} {m} {r.size}"]
    lines += [f"{a} {b} {x:.17g}" for a, b, x in zip(r, c, v)]
    ours, ref = both(tmp_path, "\n".join(lines) + "\n")
    same_bytes(ours, ref)


def test_duplicates_kept_as_the_reference_keeps_them(tmp_path):
    _need_ref()
    text = """%%MatrixMarket matrix coordinate real general
3 3 6
1 2 1
1 2 2
3 1 5
1 2 3
3 1 -5
2 2 4
"""
    ours, ref = both(tmp_path, text)
    assert ours[:9] == ref[:9] and ours[16:88] == ref[16:88]
    ro, co, rpo, colo, valo = split(ours)
    rr, cr, rpr, colr, valr = split(ref)
    assert (ro, co) == (rr, cr)
    assert np.array_equal(rpo, rpr) and np.array_equal(colo, colr)
    for i in range(ro):
        for j in np.unique(colo[rpo[i]:rpo[i + 1]]):
            a = sorted(valo[rpo[i]:rpo[i + 1]][colo[rpo[i]:rpo[i + 1]] == j])
            b = sorted(valr[rpr[i]:rpr[i + 1]][colr[rpr[i]:rpr[i + 1]] == j])
            assert a == b
