"""CPU restatement of the spy-plot segmentation — TEST INFRASTRUCTURE ONLY.

Only tests/ may import this module, as the checker of libocean.so's
segmentation records (the ``segmentation`` section of the stats JSON). The
product path never calls it.

Restates kernels/Segmentation.cuh of the reference step by step:
  * density map: A's nonzeros counted per (row // tile_rows, col // tile_cols)
    tile, grid at most grid_max per side (Segmentation.cuh:79-104, 404-417);
  * hot tiles: density >= mean + k * stddev and > 0, label = tile index
    (Segmentation.cuh:108-124, 446-476);
  * 4-connected components by min-label propagation, then pointer jumping
    (Segmentation.cuh:126-183, 478-514);
  * dominant label per grid row (Segmentation.cuh:185-246);
  * row bands by run-length encoding, short bands merged into the previous
    one, distinct labels counted (Segmentation.cuh:527-575);
  * per-band reductions and the class rule (Segmentation.cuh:248-384).
Two points are fixed where the reference leaves them to thread timing, and the
library does the same: labels propagate Jacobi style (every round reads the
previous round's labels), which converges to the reference's labels (smallest
tile index of the component) with a deterministic round count; and a tie of
the dominant label goes to the label with the earlier hash slot
(label * 2654435761 mod 2^32 mod grid_w), then the smaller label — the
reference's table order when no two labels of the row share a slot.
Every floating-point operation is rounded on its own, as in the library.

Parity is unpinned against reference outputs: the reference's segmentation
needs its own GPU build and has no golden vectors. It is anchored on this
restatement and on hand-checked cases in tests/test_oracle_segmentation.py.
"""
from __future__ import annotations

import math

import numpy as np

NONE = 0xFFFFFFFF
CLASS_NAMES = ["SPARSE_UNIFORM", "DENSE", "POWER_LAW", "BANDED"]


def row_stats(A, B):
    """Per row of A: products, smallest/largest output column (NONE/0 when the
    row has no product), entries of A, longest referenced B row
    (kernels/Analysis.cuh:52-97)."""
    arp = np.asarray(A.rowptr, np.int64)
    brp = np.asarray(B.rowptr, np.int64)
    acol = np.asarray(A.col, np.int64)
    bcol = np.asarray(B.col, np.int64)
    blen = brp[1:] - brp[:-1]
    anz = (arp[1:] - arp[:-1]).astype(np.int64)
    rows = A.rows
    L = blen[acol]                       # length of the B row each A entry references
    nonempty = L > 0
    first = np.where(nonempty, bcol[np.minimum(brp[acol], max(len(bcol) - 1, 0))] if len(bcol) else 0, NONE)
    last = np.where(nonempty, bcol[np.maximum(brp[acol + 1] - 1, 0)] if len(bcol) else 0, 0)
    row_of = np.repeat(np.arange(rows), anz)
    prod = np.zeros(rows, np.int64)
    np.add.at(prod, row_of, L)
    lo = np.full(rows, NONE, np.int64)
    np.minimum.at(lo, row_of, np.where(nonempty, first, NONE))
    hi = np.zeros(rows, np.int64)
    np.maximum.at(hi, row_of, np.where(nonempty, last, 0))
    maxb = np.zeros(rows, np.int64)
    np.maximum.at(maxb, row_of, L)
    return prod, lo, hi, anz, maxb


def segment(A, B, grid_max=256, hot_k=2.0, min_segment_rows=1024, cc_max_iters=32, expansion_threshold=8):
    """The segmentation of A (multiplied by B) as a dict shaped like the
    library's stats section (timings left out)."""
    rows, bcols = A.rows, B.cols
    out = {"segments": []}
    if rows == 0 or bcols == 0:
        return out
    gmax = min(max(8, grid_max), 4096)
    gh, gw = min(gmax, rows), min(gmax, bcols)
    tr_, tc_ = -(-rows // gh), -(-bcols // gw)
    out.update(grid_h=gh, grid_w=gw, tile_rows=tr_, tile_cols=tc_)
    arp = np.asarray(A.rowptr, np.int64)
    acol = np.asarray(A.col, np.int64)
    row_of = np.repeat(np.arange(rows), arp[1:] - arp[:-1])
    ty = np.minimum(row_of // tr_, gh - 1)
    tx = np.minimum(acol // tc_, gw - 1)
    dens = np.bincount(ty * gw + tx, minlength=gh * gw).astype(np.int64)
    tiles = gh * gw
    sa, sb = int(dens.sum()), int((dens * dens).sum())
    mean = float(sa) / float(tiles)
    var = float(sb) / float(tiles) - mean * mean
    var = max(var, 0.0)
    sd = math.sqrt(var)
    thresh = mean + hot_k * sd
    out["density_mean"], out["density_stddev"] = mean, sd
    idx = np.arange(tiles, dtype=np.int64)
    lab = np.where((dens.astype(np.float64) >= thresh) & (dens > 0), idx, NONE).reshape(gh, gw)

    it = 0
    while it < max(0, cc_max_iters):
        p = np.full((gh + 2, gw + 2), NONE, np.int64)
        p[1:-1, 1:-1] = lab
        best = np.minimum.reduce([lab, p[1:-1, :-2], p[1:-1, 2:], p[:-2, 1:-1], p[2:, 1:-1]])
        best = np.where(lab == NONE, NONE, best)
        changed = bool((best < lab).any())
        lab = best
        if not changed:
            break
        it += 1
    flat = lab.reshape(-1)
    for _ in range(8):
        nxt = np.where(flat == NONE, NONE, flat[np.minimum(flat, tiles - 1)])
        changed = bool((nxt != flat).any())
        flat = nxt
        if not changed:
            break
    lab = flat.reshape(gh, gw)
    out["cc_iterations"] = it

    band = []
    for y in range(gh):
        hot = lab[y][lab[y] != NONE]
        if hot.size == 0:
            band.append(NONE)
            continue
        labels, counts = np.unique(hot, return_counts=True)
        slots = (labels * 2654435761 % (1 << 32)) % gw
        order = sorted(range(labels.size), key=lambda i: (-int(counts[i]), int(slots[i]), int(labels[i])))
        band.append(int(labels[order[0]]))

    bands = []
    cur, cur_start = band[0], 0
    for g in range(1, gh):
        if band[g] != cur:
            s, e = cur_start * tr_, min(rows, g * tr_)
            if e > s:
                bands.append([s, e, cur])
            cur, cur_start = band[g], g
    s, e = cur_start * tr_, rows
    if e > s:
        bands.append([s, e, cur])
    merged = []
    min_rows = max(1, min_segment_rows)
    for b in bands:
        if merged and b[1] - b[0] < min_rows:
            merged[-1][1] = b[1]
        else:
            merged.append(list(b))
    uniq = []
    for b in merged:
        if b[2] != NONE and b[2] not in uniq:
            uniq.append(b[2])
    out["num_components"] = len(uniq)
    if not merged:
        merged = [[0, rows, NONE]]

    prod, lo, hi, anz, maxb = row_stats(A, B)
    prod = np.minimum(prod, NONE)
    for r0, r1, _ in merged:
        p = prod[r0:r1]
        sp = int(p.sum())
        sq = int((p.astype(object) ** 2).sum()) & ((1 << 64) - 1) if p.size else 0
        sa_ = int(anz[r0:r1].sum())
        cl = int(lo[r0:r1].min()) if r1 > r0 else NONE
        cr = int(hi[r0:r1].max()) if r1 > r0 else 0
        n = r1 - r0
        col_left = 0 if cl == NONE else cl
        mean_p = float(sp) / float(n) if n > 0 else 0.0
        var_p = 0.0
        if n > 0:
            var_p = float(sq) / float(n) - mean_p * mean_p
        var_p = max(var_p, 0.0)
        cv = math.sqrt(var_p) / mean_p if mean_p > 0.0 else 0.0
        er = float(sp) / float(sa_) if sa_ > 0 else 0.0
        span = ((cr + 1 - col_left) & 0xFFFFFFFF)
        ratio = float(span) / float(bcols) if bcols > 0 else 0.0
        density = mean_p / (float(bcols) * ratio) if ratio > 0.0 else 0.0
        cls = 0
        if 0.0 < ratio < 0.05 and mean_p > 0.0 and er >= float(expansion_threshold):
            cls = 3
        elif density >= 0.25:
            cls = 1
        elif cv >= 1.5:
            cls = 2
        out["segments"].append({
            "row_start": r0, "row_end": r1, "row_count": n, "col_left": col_left, "col_right": cr,
            "class": CLASS_NAMES[cls], "sum_products": sp, "sum_a_nnz": sa_, "mean_row_len": mean_p,
            "var_row_len": var_p, "local_er": er, "max_b_row_len": int(maxb[r0:r1].max()) if n else 0,
            "max_a_row_len": int(anz[r0:r1].max()) if n else 0,
        })
    return out
