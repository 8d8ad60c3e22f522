"""The `spgemm` driver: the reference's argv and JSON config surface
(src/main.cu:11-83), .hicsr input, ground-truth comparison, stats JSON."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import HostCSR

CLI = Path(__file__).resolve().parent.parent / "research_b200" / "bin" / "spgemm"


def run(*args, timeout=300):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, timeout=timeout)


def test_usage_and_bad_files(tmp_path):
    r = run()
    assert r.returncode == 1 and "Usage" in r.stderr
    bad = tmp_path / "x.mtxd_.hicsr"
    bad.write_bytes(b"garbage" * 20)
    r = run(bad)
    assert r.returncode == 1 and "does not appear to be a CSR" in (r.stdout + r.stderr)


def test_dimension_mismatch_rejected(tmp_path):
    A = M.rect_poisson(20, 30, 3.0, seed=1)
    pa, pb = tmp_path / "a.mtxd_.hicsr", tmp_path / "b.mtxd_.hicsr"
    M.write_hicsr(A, pa)
    M.write_hicsr(A, pb)
    r = run(pa, pb)
    assert r.returncode == 1 and "Incompatible" in r.stderr


@pytest.mark.gpu
def test_cli_matches_oracle_and_writes_stats(tmp_path):
    A = M.laplacian_2d(64, 64, seed=3)
    pa = tmp_path / "lap.mtxd_.hicsr"
    M.write_hicsr(A, pa)
    cp, cj, cx = O.spgemm(A, A)
    truth = HostCSR(A.rows, A.cols, cp.astype(np.uint32), cj, cx)
    pt = tmp_path / "truth.mtxd_.hicsr"
    M.write_hicsr(truth, pt)
    cfg = tmp_path / "cfg.json"
    stats = tmp_path / "stats.json"
    cfg.write_text(json.dumps({"warmup_iters": 1, "bench_iters": 2, "check_correctness": True,
                               "ground_truth_file": str(pt), "output_stats": True,
                               "stats_output_file": str(stats), "track_stage_time": True}))
    r = run(pa, cfg)
    assert r.returncode == 0, r.stderr
    assert "Comparison completed" in r.stdout
    st = json.loads(stats.read_text())
    assert st["C"]["nnz"] == int(cp[-1]) and st["gflops"] > 0 and "timing" in st


@pytest.mark.gpu
def test_cli_rejects_wrong_ground_truth(tmp_path):
    A = M.uniform_random(500, 4, seed=4)
    pa = tmp_path / "u.mtxd_.hicsr"
    M.write_hicsr(A, pa)
    pt = tmp_path / "wrong.mtxd_.hicsr"
    M.write_hicsr(A, pt)  # A is not A*A
    cfg = tmp_path / "cfg.json"
    cfg.write_text(json.dumps({"warmup_iters": 0, "bench_iters": 1, "check_correctness": True,
                               "ground_truth_file": str(pt)}))
    r = run(pa, pa, cfg)
    assert r.returncode == 1 and "different" in r.stderr
