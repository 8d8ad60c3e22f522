"""FAT workflow (reference kernels/SpGEMM.cuh:456-466, 925-1050): a short, fat
A times a tall, skinny B with few output columns gives every row its exact
upper bound min(products, span) as its slots; C equals the oracle's."""
import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import SpGEMM

pytestmark = pytest.mark.gpu


def fat_pair(rows=50, inner=20000, cols=64, per_row=400, seed=1):
    rng = np.random.default_rng(seed)
    r = np.repeat(np.arange(rows), per_row)
    c = rng.integers(0, inner, r.size)
    A = M.from_coo(rows, inner, r, c, rng.uniform(-1, 1, r.size))
    rb = np.repeat(np.arange(inner), 3)
    cb = rng.integers(0, cols, rb.size)
    B = M.from_coo(inner, cols, rb, cb, rng.uniform(-1, 1, rb.size))
    return A, B


def check(g, A, B, workflow):
    C = g.multiply(A, B)
    rp, cj, cx, ca = O.spgemm(A, B, with_abs=True)
    O.compare(C.rowptr, C.col, C.val, rp, cj, cx, ref_abs=ca)
    st = g.get_stats()
    assert st["decision"]["workflow"] == workflow
    return st


def test_fat_shape_takes_the_fat_workflow():
    A, B = fat_pair()
    st = check(SpGEMM({"output_stats": True}), A, B, 3)
    assert st["estimation"]["estimator"] == "bound" and st["estimation"]["overflow_rows"] == 0


def test_fat_workflow_can_be_switched_off_or_forced():
    A, B = fat_pair(seed=2)
    check(SpGEMM({"use_fat_workflow": False}), A, B, 0)
    R = M.rmat(12, 8, seed=3)
    check(SpGEMM({"force_workflow": 3}), R, R, 3)
