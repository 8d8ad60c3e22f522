#!/usr/bin/env python3
"""Charts from the library's stats JSON files, as SVG (no plotting library).

Same inputs, options and charts as the reference's post-processing script
(utils/plot_results.py:1-175):

  - ``gflops.svg``: GFLOP/s bar chart across matrices (``gflops`` key,
    utils/plot_results.py:42-55);
  - ``overhead_breakdown.svg``: segmentation stage times (density, threshold,
    CC, classify) stacked under the total time, and their share of the total
    (utils/plot_results.py:58-89);
  - ``spy_<matrix>.svg``: the matrix pattern with the detected segments
    overlaid, one colour per class (utils/plot_results.py:92-131).

Stats files are ``<results_dir>/<matrix>_stats.json`` as the ``spgemm``
driver writes them. The spy plot reads ``<mtx_dir>/<matrix>/<matrix>.mtx``
with the library's MatrixMarket reader (or ``<matrix>.hicsr`` beside it);
its pattern is drawn as an embedded PNG raster (one pixel per cell of a
grid over the matrix, darker with more entries) and the segments as
rectangles on top.

Usage: python -m research_b200.plot_results RESULTS_DIR --matrices a,b,c
       [--mtx-dir DIR] [--out plots]
"""
from __future__ import annotations

import argparse
import base64
import json
import struct
import sys
import zlib
from pathlib import Path
from xml.sax.saxutils import escape

import numpy as np

CLASS_COLORS = {
    "sparse_uniform": "#4c78a8",
    "dense": "#e45756",
    "power_law": "#f58518",
    "banded": "#54a24b",
}
STAGE_KEYS = [
    ("time_density_ms", "density"),
    ("time_threshold_ms", "threshold"),
    ("time_cc_ms", "CC"),
    ("time_classify_ms", "classify"),
]
STAGE_COLORS = ["#4c78a8", "#f58518", "#54a24b", "#b279a2"]
OTHER_COLOR = "#cccccc"


def load_stats(results_dir: Path, matrix: str) -> dict:
    path = results_dir / f"{matrix}_stats.json"
    if not path.exists():
        print(f"  [warn] missing {path}", file=sys.stderr)
        return {}
    with open(path) as f:
        return json.load(f)


# ----------------------------------------------------------------------------- SVG helpers
class Svg:
    def __init__(self, width: int, height: int):
        self.w, self.h = width, height
        self.items: list[str] = []

    def rect(self, x, y, w, h, fill, opacity=1.0, stroke=None, cls=None, title=None):
        extra = f' stroke="{stroke}" stroke-width="1"' if stroke else ""
        extra += f' class="{cls}"' if cls else ""
        t = f"<title>{escape(title)}</title>" if title else ""
        self.items.append(f'<rect x="{x:.2f}" y="{y:.2f}" width="{max(w, 0):.2f}" height="{max(h, 0):.2f}" '
                          f'fill="{fill}" fill-opacity="{opacity}"{extra}>{t}</rect>')

    def line(self, x1, y1, x2, y2, color="#000"):
        self.items.append(f'<line x1="{x1:.2f}" y1="{y1:.2f}" x2="{x2:.2f}" y2="{y2:.2f}" stroke="{color}"/>')

    def text(self, x, y, s, size=11, anchor="middle", rotate=None):
        tr = f' transform="rotate({rotate} {x:.2f} {y:.2f})"' if rotate is not None else ""
        self.items.append(f'<text x="{x:.2f}" y="{y:.2f}" font-family="sans-serif" font-size="{size}" '
                          f'text-anchor="{anchor}"{tr}>{escape(str(s))}</text>')

    def image_png(self, x, y, w, h, png: bytes):
        data = base64.b64encode(png).decode()
        self.items.append(f'<image x="{x}" y="{y}" width="{w}" height="{h}" preserveAspectRatio="none" '
                          f'style="image-rendering:pixelated" href="data:image/png;base64,{data}"/>')

    def save(self, path: Path):
        body = "\n".join(self.items)
        path.write_text(f'<svg xmlns="http://www.w3.org/2000/svg" width="{self.w}" height="{self.h}" '
                        f'viewBox="0 0 {self.w} {self.h}">\n<rect width="100%" height="100%" fill="#fff"/>\n'
                        f"{body}\n</svg>\n")


def _nice_max(v: float) -> float:
    if v <= 0:
        return 1.0
    e = 10 ** np.floor(np.log10(v))
    for m in (1, 2, 2.5, 5, 10):
        if m * e >= v:
            return float(m * e)
    return float(10 * e)


def _axes(svg: Svg, x0, y0, w, h, ymax, ylabel, title, ticks=5):
    svg.line(x0, y0 + h, x0 + w, y0 + h)
    svg.line(x0, y0, x0, y0 + h)
    for i in range(ticks + 1):
        v = ymax * i / ticks
        y = y0 + h - h * i / ticks
        svg.line(x0 - 4, y, x0, y)
        svg.text(x0 - 6, y + 4, f"{v:g}", size=10, anchor="end")
    svg.text(x0 - 44, y0 + h / 2, ylabel, size=11, rotate=-90)
    svg.text(x0 + w / 2, y0 - 10, title, size=13)


def _bars(svg: Svg, x0, y0, w, h, names, stacks, ymax, labels=None):
    """stacks: list over bars of [(value, colour, tooltip), ...] bottom-up."""
    n = max(len(names), 1)
    slot = w / n
    bw = slot * 0.6
    for i, name in enumerate(names):
        bx = x0 + slot * i + (slot - bw) / 2
        base = 0.0
        for v, color, tip in stacks[i]:
            hh = h * v / ymax if ymax > 0 else 0
            svg.rect(bx, y0 + h - h * base / ymax - hh, bw, hh, color, cls="bar", title=f"{name} {tip}: {v:.4g}")
            base += v
        if labels:
            svg.text(bx + bw / 2, y0 + h - h * base / ymax - 4, labels[i], size=10)
        svg.text(bx + bw / 2, y0 + h + 14, name, size=10)


def plot_gflops(stats_by_matrix: dict, out: Path) -> None:
    names = list(stats_by_matrix)
    vals = [float(stats_by_matrix[m].get("gflops", 0.0)) for m in names]
    svg = Svg(700, 400)
    x0, y0, w, h = 70, 40, 610, 310
    ymax = _nice_max(max(vals) if vals else 1.0)
    _axes(svg, x0, y0, w, h, ymax, "GFLOPS", "Ocean SpGEMM (block-segmented) - GFLOPS")
    _bars(svg, x0, y0, w, h, names, [[(v, "#4c78a8", "gflops")] for v in vals], ymax,
          labels=[f"{v:.1f}" for v in vals])
    svg.save(out)


def plot_overhead(stats_by_matrix: dict, out: Path) -> None:
    names = list(stats_by_matrix)
    totals = np.array([float(stats_by_matrix[m].get("total_time", 0.0)) for m in names])
    stage = np.array([[float(stats_by_matrix[m].get("segmentation", {}).get(k, 0.0)) for k, _ in STAGE_KEYS]
                      for m in names]).reshape(len(names), len(STAGE_KEYS))
    seg_total = stage.sum(axis=1) if len(names) else np.zeros(0)
    other = np.maximum(totals - seg_total, 0.0)
    svg = Svg(1200, 450)
    # absolute stage breakdown
    x0, y0, w, h = 70, 40, 480, 330
    ymax = _nice_max(float(np.max(seg_total + other)) if len(names) else 1.0)
    _axes(svg, x0, y0, w, h, ymax, "time (ms / iter)", "Stage breakdown (absolute)")
    stacks = []
    for i in range(len(names)):
        st = [(float(stage[i, j]), STAGE_COLORS[j], STAGE_KEYS[j][1]) for j in range(len(STAGE_KEYS))]
        st.append((float(other[i]), OTHER_COLOR, "other SpGEMM"))
        stacks.append(st)
    _bars(svg, x0, y0, w, h, names, stacks, ymax)
    for j, (label, color) in enumerate([(k[1], c) for k, c in zip(STAGE_KEYS, STAGE_COLORS)] +
                                       [("other SpGEMM", OTHER_COLOR)]):
        svg.rect(x0 + w - 110, y0 + 6 + 16 * j, 10, 10, color, cls="legend")
        svg.text(x0 + w - 95, y0 + 15 + 16 * j, label, size=10, anchor="start")
    # segmentation share of the total
    pct = np.where(totals > 0, 100.0 * seg_total / np.where(totals > 0, totals, 1.0), 0.0)
    x1 = 680
    pmax = _nice_max(float(pct.max()) if len(pct) and pct.max() > 0 else 1.0)
    _axes(svg, x1, y0, w, h, pmax, "segmentation overhead (% of total)", "Segmentation overhead vs total")
    _bars(svg, x1, y0, w, h, names, [[(float(p), "#e45756", "segmentation %")] for p in pct], pmax,
          labels=[f"{p:.1f}%" for p in pct])
    svg.save(out)


# ----------------------------------------------------------------------------- spy plot
def png_gray(img: np.ndarray) -> bytes:
    """8-bit grayscale PNG of a 2-D uint8 array (stored rows, zlib, CRCs)."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    hgt, wid = img.shape
    raw = b"".join(b"\x00" + img[r].tobytes() for r in range(hgt))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", wid, hgt, 8, 0, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(raw, 9)) + chunk(b"IEND", b""))


def spy_raster(rows: int, cols: int, r: np.ndarray, c: np.ndarray, px: int = 700) -> np.ndarray:
    """Occupancy raster: cell (i, j) of a px-wide grid is darker with more entries."""
    gh = max(1, min(px, rows))
    gw = max(1, min(px, cols))
    ri = (r.astype(np.int64) * gh // max(rows, 1)).clip(0, gh - 1)
    ci = (c.astype(np.int64) * gw // max(cols, 1)).clip(0, gw - 1)
    cnt = np.bincount(ri * gw + ci, minlength=gh * gw).reshape(gh, gw).astype(np.float64)
    img = np.full((gh, gw), 255, np.uint8)
    nz = cnt > 0
    if nz.any():
        # log-scaled darkness, any occupied cell at least mid-grey
        lv = np.log1p(cnt[nz]) / np.log1p(cnt.max())
        img[nz] = (160 - 160 * lv).astype(np.uint8)
    return img


def _load_pattern(path: Path):
    from research_b200 import matrices as M

    if path.suffix == ".hicsr":
        A = M.read_hicsr(str(path))
    else:
        A = M.read_mtx(str(path))
    rp = np.asarray(A.rowptr, np.int64)
    rows_idx = np.repeat(np.arange(A.rows, dtype=np.int64), np.diff(np.append(rp[:A.rows], A.nnz)))
    return A.rows, A.cols, rows_idx, np.asarray(A.col, np.int64)


def plot_spy(matrix: str, stats: dict, mtx_path: Path, out: Path) -> None:
    if not mtx_path.exists():
        alt = mtx_path.with_suffix(".hicsr")
        if alt.exists():
            mtx_path = alt
        else:
            print(f"  [warn] missing {mtx_path}; skipping spy plot for {matrix}", file=sys.stderr)
            return
    print(f"  reading {mtx_path} ...")
    rows, cols, r, c = _load_pattern(mtx_path)
    img = spy_raster(rows, cols, r, c)
    side = 700
    scale = side / max(rows, cols, 1)
    pw, ph = max(1.0, cols * scale), max(1.0, rows * scale)
    svg = Svg(int(pw) + 100, int(ph) + 80)
    x0, y0 = 50, 40
    svg.image_png(x0, y0, f"{pw:.2f}", f"{ph:.2f}", png_gray(img))
    svg.rect(x0, y0, pw, ph, "none", stroke="#000")
    svg.text(x0 + pw / 2, y0 - 12, f"{matrix}  (segments overlaid)", size=13)
    seen = []
    for seg in stats.get("segmentation", {}).get("segments", []):
        cls = seg.get("class", "sparse_uniform")
        color = CLASS_COLORS.get(cls.lower(), "#888888")  # the stats spell classes in capitals
        sx = x0 + seg["col_left"] * scale
        sy = y0 + seg["row_start"] * scale
        sw = max(seg["col_right"] - seg["col_left"], 1) * scale
        sh = max(seg["row_end"] - seg["row_start"], 1) * scale
        svg.rect(sx, sy, sw, sh, color, opacity=0.18, stroke=color, cls="segment",
                 title=f"{cls}: rows {seg['row_start']}-{seg['row_end']}, cols {seg['col_left']}-{seg['col_right']}")
        if cls not in seen:
            seen.append(cls)
    for j, cls in enumerate(seen):
        svg.rect(x0 + pw - 120, y0 + 8 + 16 * j, 10, 10, CLASS_COLORS.get(cls.lower(), "#888888"), cls="legend")
        svg.text(x0 + pw - 105, y0 + 17 + 16 * j, cls, size=10, anchor="start")
    svg.save(out)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("results_dir", type=Path)
    ap.add_argument("--matrices", required=True, help="comma-separated, e.g. 144,road_usa,cant,belgium_osm")
    ap.add_argument("--mtx-dir", type=Path, default=None, help="directory containing <name>/<name>.mtx for spy plots")
    ap.add_argument("--out", type=Path, default=Path("plots"))
    args = ap.parse_args(argv)

    args.out.mkdir(parents=True, exist_ok=True)
    matrices = [m.strip() for m in args.matrices.split(",") if m.strip()]
    stats_by_matrix = {}
    for m in matrices:
        s = load_stats(args.results_dir, m)
        if s:
            stats_by_matrix[m] = s
    if not stats_by_matrix:
        print("no stats files found", file=sys.stderr)
        return 1
    print("rendering gflops.svg ...")
    plot_gflops(stats_by_matrix, args.out / "gflops.svg")
    print("rendering overhead_breakdown.svg ...")
    plot_overhead(stats_by_matrix, args.out / "overhead_breakdown.svg")
    if args.mtx_dir is not None:
        for m, s in stats_by_matrix.items():
            print(f"rendering spy_{m}.svg ...")
            plot_spy(m, s, args.mtx_dir / m / f"{m}.mtx", args.out / f"spy_{m}.svg")
    print(f"done -> {args.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
