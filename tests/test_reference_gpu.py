"""The reference's own CUDA build (oracle/_ref/spgemm_ref, compiled from the
reference sources by `make -C oracle refbin`) run on the 2D Laplacian 256x256
C = A*A input, with its ground-truth comparison (src/CSR.cpp:252-335) pointed at
the CPU oracle's C. This pins the oracle to the reference's actual output
(exact row offsets and column ids, values within the reference's 1e-4 hard
limit) and records the reference's GFLOP/s beside this library's on the same
input. Only this input is run: its reference path (ultra-sparse workflow, ESC
kernel of size 32, CUB scans, copy) was read and has no unbounded waits."""
import json
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import DeviceCSR, HostCSR, SpGEMM

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref" / "spgemm_ref"

pytestmark = pytest.mark.gpu


def test_reference_build_agrees_with_oracle_on_laplacian(tmp_path):
    if not REF.exists():
        pytest.skip("reference driver not built (make -C oracle refbin needs the reference source tree)")
    A = M.laplacian_2d(256, 256, seed=0)
    pa = tmp_path / "lap256.mtxd_.hicsr"
    M.write_hicsr(A, pa)
    cp, cj, cx = O.spgemm(A, A)
    pt = tmp_path / "truth.mtxd_.hicsr"
    M.write_hicsr(HostCSR(A.rows, A.cols, cp.astype(np.uint32), cj, cx), pt)
    stats = tmp_path / "ref_stats.json"
    cfg = tmp_path / "bench.json"
    cfg.write_text(json.dumps({"warmup_iters": 10, "bench_iters": 10, "check_correctness": True,
                               "ground_truth_file": str(pt), "output_stats": True,
                               "stats_output_file": str(stats), "print_info": False,
                               "track_stage_time": False}))
    r = subprocess.run([str(REF), str(pa), str(cfg)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Comparison completed" in r.stdout
    ref = json.loads(stats.read_text())
    assert ref["C"]["nnz"] == int(cp[-1])
    # this library on the same input, same iteration counts
    g = SpGEMM({"track_stage_time": False})
    dA = DeviceCSR.from_host(A)
    ms = []
    for i in range(20):
        C = g.multiply(dA, dA)
        if i >= 10:
            ms.append(g.stage_ms("total"))
        C.free()
    ours = 2.0 * 1629192 / (sum(ms) / len(ms)) / 1e6
    rec = {"input": "laplacian 256x256, C=A*A", "reference_gflops": ref["gflops"],
           "reference_ms": ref["total_time"], "reference_workflow": ref["decision"]["workflow"],
           "ours_gflops": ours, "ours_ms": sum(ms) / len(ms)}
    print(json.dumps(rec))
    out = os.environ.get("OCEAN_RECORD_DIR")
    if out:
        Path(out).mkdir(parents=True, exist_ok=True)
        (Path(out) / "reference_gpu_laplacian.json").write_text(json.dumps(rec) + "\n")
