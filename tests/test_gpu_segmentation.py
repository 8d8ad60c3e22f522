"""Spy-plot segmentation on the GPU (use_segmented_workflow): the records in
the stats JSON equal the CPU restatement field by field (timings aside), and
the product C is unchanged by the extra pass."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import segmentation as S
from research_b200 import matrices as M
from research_b200.ocean import SpGEMM

pytestmark = pytest.mark.gpu

FIELDS = ["grid_h", "grid_w", "tile_rows", "tile_cols", "density_mean", "density_stddev", "num_components",
          "cc_iterations"]


def two_blocks_and_tie():
    # two dense blocks, plus two equal hot groups side by side in one grid row
    r, c = [], []
    for base in (0, 8):
        for i in range(4):
            for j in range(4):
                r.append(base + i)
                c.append(base + j)
    for i in range(12, 14):
        for j in (0, 1, 6, 7):
            r.append(i)
            c.append(j)
    return M.from_coo(16, 16, np.array(r), np.array(c), np.ones(len(r)))


def cases():
    yield "two_blocks_tie", two_blocks_and_tie(), None, dict(segmentation_grid_max=8,
                                                              segmentation_min_segment_rows=1)
    yield "tiny_rows", M.uniform_random(5, 3, seed=1), None, {}
    yield "banded", M.banded(1 << 18, 16, 16, seed=2), None, {}
    yield "dense", M.uniform_random(2000, 200, seed=3), None, {}
    yield "uniform", M.uniform_random(100000, 8, seed=4), None, {}
    yield "rmat16", M.rmat(16, 8, seed=5), None, {}
    yield "blocks", M.block_diagonal(50000, 256, 8, seed=6), None, dict(segmentation_min_segment_rows=64)
    A = M.rect_poisson(3000, 9000, 12.0, seed=7)
    yield "rect", A, M.transpose(A), dict(segmentation_grid_max=64, segmentation_hot_threshold_k=1.0)
    yield "laplacian_k0", M.laplacian_2d(300, 200), None, dict(segmentation_hot_threshold_k=0.0,
                                                               segmentation_cc_max_iters=4)
    yield "rmat_wide_grid", M.rmat(14, 8, seed=8), None, dict(segmentation_grid_max=2048,
                                                              segmentation_min_segment_rows=16)


@pytest.mark.parametrize("name,A,B,cfg", list(cases()), ids=[c[0] for c in cases()])
def test_segmentation_records_match_restatement(name, A, B, cfg):
    B = A if B is None else B
    config = {"use_segmented_workflow": True, "output_stats": True, **cfg}
    g = SpGEMM(config)
    C = g.multiply(A, B)
    got = g.get_stats()["segmentation"]
    want = S.segment(A, B, grid_max=cfg.get("segmentation_grid_max", 256),
                     hot_k=cfg.get("segmentation_hot_threshold_k", 2.0),
                     min_segment_rows=cfg.get("segmentation_min_segment_rows", 1024),
                     cc_max_iters=cfg.get("segmentation_cc_max_iters", 32))
    for f in FIELDS:
        assert got[f] == want[f], f
    assert len(got["segments"]) == len(want["segments"])
    for a, b in zip(got["segments"], want["segments"]):
        assert a == b
    for t in ("time_density_ms", "time_threshold_ms", "time_cc_ms", "time_classify_ms"):
        assert got[t] >= 0.0
    rp, rj, rx, ra = O.spgemm(A, B, with_abs=True)
    O.compare(C.rowptr, C.col, C.val, rp, rj, rx, ref_abs=ra)


def test_segmentation_with_64bit_row_offsets_and_off_by_default():
    A = M.rmat(13, 8, seed=9).widened()
    g = SpGEMM({"use_segmented_workflow": True})
    g.multiply(A, A)
    got = g.get_stats()["segmentation"]["segments"]
    assert got == S.segment(A, A)["segments"]
    g2 = SpGEMM({})
    g2.multiply(A, A)
    assert "segmentation" not in g2.get_stats()
