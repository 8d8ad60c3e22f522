"""MatrixMarket reading with the reference converter's rules
(utils/convert.cpp:83-240) and the .mtx -> .hicsr converter."""
import numpy as np
import pytest

from research_b200 import matrices as M
from research_b200.convert import main as convert_main


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return p


def test_general_real_with_comments_and_blank_lines(tmp_path):
    p = write(tmp_path, "a.mtx", """%%MatrixMarket matrix coordinate real general
% a comment
3 4 5

1 1 1.5
3 4 -2
1 3 0.25
% another comment
2 2 7
3 1 1e-3
""")
    m = M.read_mtx(p)
    assert (m.rows, m.cols, m.nnz) == (3, 4, 5)
    assert list(m.rowptr) == [0, 2, 3, 5]
    assert list(m.col) == [0, 2, 1, 0, 3]
    assert list(m.val) == [1.5, 0.25, 7.0, 1e-3, -2.0]


def test_symmetric_pattern_mirrors_off_diagonal_entries(tmp_path):
    p = write(tmp_path, "s.mtx", """%%MatrixMarket matrix coordinate pattern symmetric
3 3 3
1 1
2 1
3 2
""")
    m = M.read_mtx(p)
    assert m.nnz == 5
    assert list(m.rowptr) == [0, 2, 4, 5]
    assert list(m.col) == [0, 1, 0, 2, 1]
    assert np.all(m.val == 1.0)


def test_integer_hermitian_complex_and_duplicates(tmp_path):
    p = write(tmp_path, "h.mtx", """%%MatrixMarket matrix coordinate complex Hermitian
2 2 3
1 1 2 0
2 1 3 -4
2 1 5 1
""")
    m = M.read_mtx(p)
    # real parts; (2,1) mirrored to (1,2); the duplicate (2,1) kept in file order
    assert list(m.rowptr) == [0, 3, 5]
    assert list(m.col) == [0, 1, 1, 0, 0]
    assert list(m.val) == [2.0, 3.0, 5.0, 3.0, 5.0]
    q = write(tmp_path, "i.mtx", "%%MatrixMarket matrix coordinate integer general\n2 2 1\n2 2 9\n")
    assert list(M.read_mtx(q).val) == [9.0]


@pytest.mark.parametrize("text,msg", [
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "coordinate"),
    ("%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 1\n", "symmetric"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", "Row index"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 0 1\n", "Column index"),
    ("%%MatrixMarket matrix coordinate text general\n2 2 1\n1 1 1\n", "data type"),
])
def test_rejected_files(tmp_path, text, msg):
    with pytest.raises(ValueError, match=msg):
        M.read_mtx(write(tmp_path, "bad.mtx", text))


def test_converter_round_trip(tmp_path):
    A = M.uniform_random(200, 6, seed=3)
    r = np.repeat(np.arange(A.rows), np.diff(A.rowptr.astype(np.int64)))
    lines = ["%%MatrixMarket matrix coordinate real general", f"{A.rows} {A.cols} {A.nnz}"]
    lines += [f"{i + 1} {j + 1} {float(v)!r}" for i, j, v in zip(r, A.col, A.val)]
    src = write(tmp_path, "u.mtx", "\n".join(lines) + "\n")
    dst = tmp_path / "u.hicsr"
    assert convert_main([str(src), str(dst)]) == 0
    back = M.read_hicsr(dst)
    assert np.array_equal(back.rowptr, A.rowptr) and np.array_equal(back.col, A.col)
    assert np.array_equal(back.val, A.val)
