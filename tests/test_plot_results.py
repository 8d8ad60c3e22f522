"""Stats charts (research_b200.plot_results): the three outputs of the
reference's post-processing script, checked through their SVG structure."""
import json
import struct
import xml.etree.ElementTree as ET
import zlib

import numpy as np
import pytest

from research_b200 import plot_results as P

NS = {"s": "http://www.w3.org/2000/svg"}


def _stats(gflops, total, seg_times=None, segments=()):
    s = {"gflops": gflops, "total_time": total}
    if seg_times is not None:
        s["segmentation"] = {"time_density_ms": seg_times[0], "time_threshold_ms": seg_times[1],
                             "time_cc_ms": seg_times[2], "time_classify_ms": seg_times[3],
                             "segments": list(segments)}
    return s


def _rects(path, cls):
    root = ET.parse(path).getroot()
    return [r for r in root.iter("{http://www.w3.org/2000/svg}rect") if r.get("class") == cls]


def _decode_png(data: bytes) -> np.ndarray:
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = None
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert crc == zlib.crc32(tag + body) & 0xFFFFFFFF
        if tag == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    assert len(raw) == h * (w + 1)
    rows = [raw[r * (w + 1) + 1:(r + 1) * (w + 1)] for r in range(h)]
    return np.frombuffer(b"".join(rows), np.uint8).reshape(h, w)


def test_gflops_and_overhead_charts(tmp_path):
    res = tmp_path / "results"
    res.mkdir()
    stats = {"a": _stats(100.0, 10.0, (1.0, 0.5, 2.0, 0.5)), "b": _stats(50.0, 4.0, (0.0, 0.0, 0.0, 1.0)),
             "c": _stats(25.0, 2.0)}
    for k, v in stats.items():
        (res / f"{k}_stats.json").write_text(json.dumps(v))
    out = tmp_path / "plots"
    assert P.main([str(res), "--matrices", "a,b,c,missing", "--out", str(out)]) == 0
    bars = _rects(out / "gflops.svg", "bar")
    assert len(bars) == 3
    hts = [float(b.get("height")) for b in bars]
    assert hts[0] == pytest.approx(2 * hts[1]) and hts[1] == pytest.approx(2 * hts[2])
    ob = _rects(out / "overhead_breakdown.svg", "bar")
    # 3 matrices x (4 stages + other) stacked, then 3 percentage bars
    assert len(ob) == 3 * 5 + 3
    stack_a = [float(r.get("height")) for r in ob[:5]]
    assert sum(stack_a[:4]) == pytest.approx(0.4 * sum(stack_a))  # 4 of 10 ms are segmentation
    pct = [float(r.get("height")) for r in ob[15:]]
    assert pct[0] == pytest.approx(pct[1] * 40 / 25)  # 40% and 25%
    assert pct[2] == 0.0


def test_no_stats_is_an_error(tmp_path):
    assert P.main([str(tmp_path), "--matrices", "x", "--out", str(tmp_path / "o")]) == 1


def test_spy_with_segments(tmp_path):
    res = tmp_path / "results"
    (res).mkdir()
    mdir = tmp_path / "mtx" / "m"
    mdir.mkdir(parents=True)
    # 40 x 40 pattern: an 8 x 8 dense block at the top left and a diagonal
    ent = [(i, j) for i in range(8) for j in range(8)] + [(i, i) for i in range(8, 40)]
    lines = ["%%MatrixMarket matrix coordinate real general", "40 40 %d" % len(ent)]
    lines += [f"{i + 1} {j + 1} 1.0" for i, j in ent]
    (mdir / "m.mtx").write_text("\n".join(lines) + "\n")
    segs = [{"row_start": 0, "row_end": 8, "col_left": 0, "col_right": 8, "class": "dense"},
            {"row_start": 8, "row_end": 40, "col_left": 8, "col_right": 40, "class": "banded"}]
    (res / "m_stats.json").write_text(json.dumps(_stats(1.0, 1.0, (0.1, 0.1, 0.1, 0.1), segs)))
    out = tmp_path / "plots"
    assert P.main([str(res), "--matrices", "m", "--mtx-dir", str(tmp_path / "mtx"), "--out", str(out)]) == 0
    svg = out / "spy_m.svg"
    rects = _rects(svg, "segment")
    assert len(rects) == 2
    assert float(rects[0].get("width")) == pytest.approx(float(rects[1].get("width")) * 8 / 32)
    root = ET.parse(svg).getroot()
    img = next(root.iter("{http://www.w3.org/2000/svg}image"))
    href = img.get("href")
    import base64
    raster = _decode_png(base64.b64decode(href.split(",", 1)[1]))
    assert raster.shape == (40, 40)  # one cell per row/column for a small matrix
    occ = raster < 255
    want = np.zeros((40, 40), bool)
    for i, j in ent:
        want[i, j] = True
    assert np.array_equal(occ, want)


def test_spy_raster_scales_down():
    r = np.array([0, 999, 500, 500])
    c = np.array([0, 1999, 1000, 1000])
    img = P.spy_raster(1000, 2000, r, c, px=100)
    assert img.shape == (100, 100)
    assert img[0, 0] < 255 and img[99, 99] < 255
    assert img[50, 50] < img[0, 0]  # two entries in that cell: darker
    assert (img < 255).sum() == 3


@pytest.mark.gpu
def test_charts_from_library_stats(tmp_path):
    """Stats JSON of a real multiply with segmentation on, written as the
    driver writes it, charted with every segment drawn."""
    from research_b200 import matrices as M
    from research_b200.ocean import SpGEMM

    res = tmp_path / "results"
    res.mkdir()
    mdir = tmp_path / "mtx"
    names = []
    for name, A in (("banded", M.banded(1 << 15, 32, 12, seed=3)), ("rmat", M.rmat(14, 8, seed=4))):
        g = SpGEMM({"use_segmented_workflow": True, "segmentation_min_segment_rows": 128})
        g.multiply(A, A)
        st = g.get_stats()
        (res / f"{name}_stats.json").write_text(json.dumps(st))
        (mdir / name).mkdir(parents=True)
        M.write_hicsr(A, mdir / name / f"{name}.hicsr")
        names.append((name, st))
    out = tmp_path / "plots"
    assert P.main([str(res), "--matrices", ",".join(n for n, _ in names), "--mtx-dir", str(mdir),
                   "--out", str(out)]) == 0
    assert len(_rects(out / "gflops.svg", "bar")) == 2
    for name, st in names:
        segs = st["segmentation"]["segments"]
        assert len(segs) > 0
        assert len(_rects(out / f"spy_{name}.svg", "segment")) == len(segs)
