"""Multi-process (world size 2, gloo, CPU) checks of the bench harness's
replica path: process-group setup, max-over-ranks timing, the barrier, and
the reference arm under torchrun (rank 0 alone works and prints one line).

The multiply itself does not shard (one independent replica per GPU, no
data-path collective), so these are the only collective steps there are."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist

    w, r, _ = bench.dist_setup()
    assert (w, r) == (world, rank)
    assert dist.get_backend() == "gloo"
    bench.barrier(w)
    # each rank reports its own elapsed time; every rank must see the largest
    got = bench.max_over_ranks(10.0 + 7.5 * rank, w)
    bench.barrier(w)
    Path(out_dir, f"rank{rank}.json").write_text(json.dumps({"max": got}))
    dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        d = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert d["max"] == pytest.approx(10.0 + 7.5 * (world - 1))


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.25, 1) == 3.25
    bench.barrier(1)  # no process group: must not raise


def test_reference_arm_under_torchrun(tmp_path):
    """`bench.py --impl reference` launched as 2 ranks: exactly one JSON line,
    from rank 0, and every rank exits 0."""
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "2"
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--workload", "laplacian256",
           "--steps", "1", "--warmup", "3"]
    p = subprocess.run(cmd, cwd=str(tmp_path), env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-4000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port"
