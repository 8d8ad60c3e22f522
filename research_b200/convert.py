"""MatrixMarket (.mtx) to the reference's binary CSR format (.hicsr), as the
reference's converter does (utils/convert.cpp:292-315).

    python -m research_b200.convert input.mtx output.hicsr
"""
from __future__ import annotations

import sys

from .matrices import read_mtx, write_hicsr


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2:
        print("usage: python -m research_b200.convert input.mtx output.hicsr", file=sys.stderr)
        return 2
    src, dst = argv
    print(f"Loading MTX file: {src}")
    m = read_mtx(src)
    print(f"  Matrix dimensions: {m.rows} x {m.cols}")
    print(f"  Non-zeros: {m.nnz}")
    print(f"Writing CSR to file: {dst}")
    write_hicsr(m, dst)
    print("Conversion complete!")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
