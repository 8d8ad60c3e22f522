"""Segment-driven dispatch (use_segment_dispatch): the rows of each spy-plot
segment take the class policy configured for the segment's class. Checked
against a CPU restatement of the class rules applied row by row with the
segments the library reported, and the product against the FP64 oracle."""
from collections import Counter

import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M

from test_gpu_parity import check, multiply_device

pytestmark = pytest.mark.gpu

SEG_KEYS = ["sparse_uniform", "dense", "power_law", "banded"]
SEG_NAMES = ["SPARSE_UNIFORM", "DENSE", "POWER_LAW", "BANDED"]


def _rows_of(m):
    return np.repeat(np.arange(m.rows), np.diff(m.rowptr.astype(np.int64)[:m.rows + 1]))


def mixed():
    """Banded rows, then dense rows in their own column window, then R-MAT rows."""
    nb, nd, nr = 65536, 4096, 16384
    n = nb + nd + nr
    Bd = M.banded(nb, 16, 16, seed=1)
    D = M.uniform_random(nd, 200, seed=3)
    R = M.rmat(14, 12, seed=2)
    r = np.concatenate([_rows_of(Bd), nb + _rows_of(D), nb + nd + _rows_of(R)])
    c = np.concatenate([Bd.col.astype(np.int64), nb + D.col.astype(np.int64), nb + nd + R.col.astype(np.int64)])
    v = np.concatenate([Bd.val, D.val, R.val])
    return M.from_coo(n, n, r, c, v)


# ---- CPU restatement of the class rules (csrc/kernels.h sym_bin_for / num_bin_for)
def policy(cfg, k=None):
    def get(key, default):
        if k is not None:
            sk = f"segment_{SEG_KEYS[k]}_{key}"
            if sk in cfg:
                return cfg[sk]
        return cfg.get(key, default)
    esc = get("esc_max_products", 128)
    hs = get("hash_s_max_scale", 1.0)
    bw = get("bitmap_words_scale", 1.0)
    d = 1 if get("prefer_direct_hash", True) else 0
    sym = dict(esc=esc, force=get("force_sym_bin", -1), hs=max(1, int(1024 * hs)), bm_m=int(2048 * bw),
               bm_l=int(8192 * bw), direct=d)
    num = dict(esc=esc, force=get("force_num_bin", -1), hs=max(1, int(512 * hs)), bm_m=int(1024 * bw),
               bm_l=int(4096 * bw), direct=d)
    return sym, num


def sym_bin(p, span, q):
    if q["force"] >= 0:
        return q["force"]
    if p <= q["esc"]:
        return 0 if p <= 32 else (1 if p <= 64 else 2)
    words = (span + 63) >> 6
    if p > 16384:
        return 6
    if p <= q["hs"]:
        return 3
    if p <= 4096:
        return 4 if (q["direct"] and span <= 8192) or words > q["bm_m"] else 6
    return 5 if (q["direct"] and span <= 32768) or words > q["bm_l"] else 6


def num_bin(n, p, span, q):
    if n == 0:
        return -1
    if q["force"] >= 0:
        return q["force"]
    if p <= q["esc"]:
        return 0 if p <= 32 else (1 if p <= 64 else 2)
    words = (span + 63) >> 6
    if n <= q["hs"]:
        return 3
    if n <= 2048:
        return 4 if (q["direct"] and span <= 4096) or words > q["bm_m"] else 6
    if n <= 4096:
        return 5 if (q["direct"] and span <= 8192) or words > q["bm_l"] else 6
    return 6


def slots_from_segments(segments, rows):
    """Dispatch slot per row: 1 + class of the first listed segment holding it, else 0."""
    slot = np.zeros(rows, np.int64)
    taken = np.zeros(rows, bool)
    for s in segments:
        a, b = s["row_start"], min(s["row_end"], rows)
        free = ~taken[a:b]
        slot[a:b][free] = 1 + SEG_NAMES.index(s["class"])
        taken[a:b] = True
    return slot


def expected_bins(A, cfg, segments):
    prod, lo, hi = O.row_stats(A, A)
    cnt = O.symbolic(A, A).astype(np.int64)
    span = hi.astype(np.int64) - lo.astype(np.int64) + 1
    slot = slots_from_segments(segments, A.rows) if segments is not None else np.zeros(A.rows, np.int64)
    pols = [policy(cfg)] + [policy(cfg, k) for k in range(4)]
    b1, b2 = Counter(), Counter()
    for i in range(A.rows):
        sp, npol = pols[slot[i]]
        p = int(prod[i])
        if p > 0:
            b1[sym_bin(p, int(span[i]), sp)] += 1
            nb = num_bin(int(cnt[i]), p, int(span[i]), npol)
            if nb >= 0:
                b2[nb] += 1
    return [b1[k] for k in range(7)], [b2[k] for k in range(7)], slot


BASE = {"force_workflow": 0, "bitmap_cache_fraction": 0.0}  # exact counts class the numeric rows; no saved bitmaps


@pytest.fixture(scope="module")
def A():
    return mixed()


def test_dispatch_without_overrides_changes_nothing(A):
    C0, st0 = multiply_device(A, A, dict(BASE))
    C1, st1 = multiply_device(A, A, dict(BASE, use_segment_dispatch=True))
    assert st1["binning_1"] == st0["binning_1"] and st1["binning_2"] == st0["binning_2"]
    assert np.array_equal(C0.rowptr, C1.rowptr) and np.array_equal(C0.col, C1.col)
    rows = st1["segment_dispatch"]["rows"]
    assert sum(rows.values()) == A.rows
    assert "segment_dispatch" not in st0


def test_segment_policies_class_their_rows(A):
    cfg = dict(BASE, use_segment_dispatch=True,
               segment_sparse_uniform_esc_max_products=32,
               segment_dense_bitmap_words_scale=0.25, segment_dense_prefer_direct_hash=False,
               segment_dense_hash_s_max_scale=0.5,
               segment_power_law_force_num_bin=6, segment_power_law_hash_s_max_scale=0.25,
               segment_banded_force_sym_bin=6)
    C, st = multiply_device(A, A, cfg)
    check(A, A, C)
    segs = st["segmentation"]["segments"]
    classes = {s["class"] for s in segs}
    assert len(classes) >= 2, classes
    b1, b2, slot = expected_bins(A, cfg, segs)
    assert st["binning_1"] == b1
    assert st["binning_2"] == b2
    rows = st["segment_dispatch"]["rows"]
    assert rows["unsegmented"] == int((slot == 0).sum())
    for k, key in enumerate(SEG_KEYS):
        assert rows[key] == int((slot == 1 + k).sum())
    # the overrides moved rows: the classes differ from the undispatched run
    _, st0 = multiply_device(A, A, dict(BASE))
    assert (st0["binning_1"], st0["binning_2"]) != (b1, b2)
    e1, e2, _ = expected_bins(A, dict(BASE), None)
    assert st0["binning_1"] == e1 and st0["binning_2"] == e2


def test_dispatch_in_the_estimated_workflow(A):
    # HLL-sized slots: the numeric classes come from the estimates, through the same per-row slots
    cfg = dict(use_segment_dispatch=True, force_workflow=1, segment_power_law_force_num_bin=6,
               segment_dense_force_num_bin=6)
    C, st = multiply_device(A, A, cfg)
    check(A, A, C)
    assert st["decision"]["workflow"] == 1

