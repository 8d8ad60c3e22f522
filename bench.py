#!/usr/bin/env python
"""SpGEMM benchmark: GFLOP/s (2 x intermediate products / s) of C = A·A on one B200.

Workload (default "rmat20"): A = square R-MAT, n = 2^20, 16 edges per vertex,
quadrant probabilities (0.57, 0.19, 0.19, 0.05), duplicate edges merged, FP64
values uniform in [-1, 1], seed 0 (synthetic, seeded; no dataset download).
C = A·A has ~2.1e10 intermediate products and ~9.7e9 entries (> 2^32, so C
carries 64-bit row pointers; ~116 GB in HBM).

One JSON line is printed by rank 0 with:
  value      device-timed throughput, inputs resident in HBM (CUDA events on the
             launching stream around K full multiplies, max over ranks);
  e2e        the same metric through the host-buffer C ABI call
             (ocean_spgemm_host): pinned host A in, C back in host memory, all
             copies inside the timed region;
  roofline   the dominant kernel's algorithmic bytes per launch / its
             event-timed duration against the measured HBM copy bandwidth;
  cpu_baseline  the CPU oracle (OpenMP Gustavson, all host cores) on a bounded
             sample of the same rows.
`--impl reference` times the CPU restatement of the path (the reference has no
CPU SpGEMM; its GPU code is the comparison the library replaces) on bounded
samples of the same workload and prints the same line with "impl": "reference".
Multi-GPU (torchrun): every rank multiplies its own replica (replicas only,
weak scaling); the value is all ranks' products over the max elapsed time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SpGEMM GFLOP/s (2*intermediate products/s), C=A*A, 1 B200"
KERNELS_PER_MULTIPLY = 1 + 7 + 3 + 7  # upper bound: analysis, symbolic classes, scan, numeric classes


# ----------------------------------------------------------------------------- workloads
def make_workload(name: str):
    from research_b200 import matrices as M
    if name == "rmat20":
        A = M.rmat(20, 16, (0.57, 0.19, 0.19, 0.05), seed=0)
        desc = ("R-MAT n=2^20, 16 edges/vertex, probs (0.57,0.19,0.19,0.05), duplicates merged, "
                "FP64 U[-1,1], seed 0; C=A*A")
        return A, A, desc
    if name == "rmat20h":
        # profiling case: every 64th heavy row (> 16384 products) of the R-MAT 2^20 workload times A
        from oracle import oracle as O
        A = M.rmat(20, 16, (0.57, 0.19, 0.19, 0.05), seed=0)
        p, _, _ = O.row_stats(A, A)
        rows = np.nonzero(p > 16384)[0][::64]
        return take_rows(A, rows), A, f"{rows.size} heavy rows of R-MAT n=2^20 (every 64th with >16384 products) times A"
    if name == "rmat20m":
        # profiling case: every 32nd heavy row with 16384 < products < 1e6 of the R-MAT 2^20 workload times A
        from oracle import oracle as O
        A = M.rmat(20, 16, (0.57, 0.19, 0.19, 0.05), seed=0)
        p, _, _ = O.row_stats(A, A)
        rows = np.nonzero((p > 16384) & (p < 1_000_000))[0][::32]
        return take_rows(A, rows), A, f"{rows.size} typical heavy rows of R-MAT n=2^20 (every 32nd with 16384 < products < 1e6) times A"
    if name == "rmat20h":
        # profiling case weighted to heavy rows: every 64th row of the R-MAT
        # 2^20 matrix (ids with six low zero bits, ~9x the mean products) times A
        A = M.rmat(20, 16, (0.57, 0.19, 0.19, 0.05), seed=0)
        rows = np.arange(0, A.rows, 64)
        return take_rows(A, rows), A, f"{rows.size} rows of R-MAT n=2^20 (every 64th, heavy-weighted) times A"
    if name == "rmat20s":
        # reduced case with the full workload's row mix (every class): a seeded
        # uniform sample of 1/64 of the rows of the R-MAT 2^20 matrix times the
        # whole matrix; its products and output entries are ~1/64 of the full
        # multiply's (a fixed stride would not do: R-MAT row weights grow with
        # the zero bits of the row id, so every 64th row is a heavy row)
        A = M.rmat(20, 16, (0.57, 0.19, 0.19, 0.05), seed=0)
        rows = np.sort(np.random.default_rng(64).choice(A.rows, A.rows // 64, replace=False))
        return take_rows(A, rows), A, f"{rows.size} rows of R-MAT n=2^20 (seeded uniform 1/64 sample) times A"
    if name.startswith("rmat"):
        sc = int(name[4:])
        A = M.rmat(sc, 16, (0.57, 0.19, 0.19, 0.05), seed=0)
        return A, A, f"R-MAT n=2^{sc}, 16 edges/vertex, seed 0; C=A*A"
    if name == "laplacian256":
        A = M.laplacian_2d(256, 256, seed=0)
        return A, A, "2D 5-point Laplacian 256x256, FP64 U[-1,1], seed 0; C=A*A"
    if name == "rect":
        A = M.rect_poisson(262144, 1048576, 12.0, seed=0)
        return A, M.transpose(A), "262144x1048576, Poisson(12)/row, uniform columns, N(0,1), seed 0; C=A*A^T"
    raise SystemExit(f"unknown workload {name}")


def compulsory_bytes(A, B, nnz_c: int) -> int:
    """Read A once + read B once + write C once (CSR: rowptr + 4 B col + 8 B val)."""
    w_c = 8 if nnz_c >= 2**32 else 4
    return (4 * (A.rows + 1) + 12 * A.nnz) + (4 * (B.rows + 1) + 12 * B.nnz) + (w_c * (A.rows + 1) + 12 * nnz_c)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("OCEAN_CLOCKS_CSV", f"/tmp/ocean_clocks_{os.getpid()}.csv"))

    def start(self):
        """Starts sampling and returns once the first sample is written, so the
        tool's own start-up (which holds the driver for a while) stays outside
        the timed region."""
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            try:
                if self.path.stat().st_size > 0:
                    break
            except OSError:
                pass
            time.sleep(0.05)
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        load = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


class NvmlSampler:
    """In-process NVML sampling of SM clocks, power and clock-event reasons
    during the timed region (a thread, one query set every 200 ms). Spawning
    nvidia-smi instead stalls the host's CUDA calls at each of its samples,
    which shows in multiplies of a millisecond or less."""
    PERIOD_S = 0.2

    def __init__(self, device: int):
        import threading
        self.device = device
        self.rows = []
        self.error = None
        self._stop = threading.Event()
        self._thread = None
        self._nv = None
        self._h = None

    def _handle(self):
        import pynvml as nv
        import torch
        p = torch.cuda.get_device_properties(self.device)
        for get in (lambda: nv.nvmlDeviceGetHandleByPciBusId(
                        f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"),
                    lambda: nv.nvmlDeviceGetHandleByUUID("GPU-" + str(p.uuid)),
                    lambda: nv.nvmlDeviceGetHandleByIndex(self.device)):
            try:
                return get()
            except Exception:
                continue
        raise RuntimeError("no NVML handle for the device")

    def _sample(self):
        nv, h = self._nv, self._h
        reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                          nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM),
                          nv.nvmlDeviceGetPowerUsage(h) / 1000.0, reasons))

    def _loop(self):
        while not self._stop.wait(self.PERIOD_S):
            try:
                self._sample()
            except Exception as e:  # keep the timing; report the sampler's failure
                self.error = str(e)
                return

    def start(self) -> bool:
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            self._nv = nv
            self._h = self._handle()
            self._sample()  # one sample before the timed region
        except Exception as e:
            self.error = str(e)
            return False
        self._thread = threading.Thread(target=self._loop, daemon=True)
        self._thread.start()
        return True

    def stop(self) -> dict:
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
            try:
                self._sample()  # and one at its end
            except Exception as e:
                self.error = self.error or str(e)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"no samples ({self.error})"]}
        nv = self._nv
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap,
                "hw_power_brake_slowdown": nv.nvmlClocksEventReasonHwPowerBrakeSlowdown}
        reasons = sorted({k for r in self.rows for k, b in bits.items() if r[3] & b})
        sm = [float(r[0]) for r in self.rows]
        mx = max(float(r[1]) for r in self.rows)
        load = [x for x in sm if x > 0.5 * mx] or sm
        out = {"sm_mhz": float(np.median(load)), "sm_max_mhz": mx, "reasons": reasons,
               "samples": len(self.rows), "power_w_max": round(max(r[2] for r in self.rows), 1),
               "source": "nvml"}
        if self.error:
            out["sampler_error"] = self.error
        return out


def clock_sampler(device: int):
    """NVML in-process sampler; nvidia-smi when NVML is not importable."""
    s = NvmlSampler(device)
    try:
        import pynvml  # noqa: F401
        return s
    except ImportError:
        return ClockSampler(device)


# ----------------------------------------------------------------------------- CPU leg
def take_rows(A, rows: np.ndarray):
    from research_b200.ocean import HostCSR
    rp = A.rowptr.astype(np.int64)
    lens = rp[rows + 1] - rp[rows]
    nrp = np.zeros(rows.size + 1, np.int64)
    np.cumsum(lens, out=nrp[1:])
    idx = np.repeat(rp[rows] - nrp[:-1], lens) + np.arange(nrp[-1])
    return HostCSR(rows.size, A.cols, nrp.astype(np.uint64), A.col[idx], A.val[idx])


def cpu_gustavson(A, B, threads: int, chunk_products: int = 300_000_000):
    """Full CPU Gustavson (symbolic + numeric) of A·B by row chunks into reused
    buffers; returns (seconds, products, per-row counts)."""
    from oracle import oracle as O
    prod, _, _ = O.row_stats(A, B, threads)
    cum = np.concatenate([[0], np.cumsum(prod.astype(np.int64))])
    counts = np.empty(A.rows, np.uint64)
    cj = cx = None
    t0 = time.perf_counter()
    r0 = 0
    while r0 < A.rows:
        r1 = int(np.searchsorted(cum, cum[r0] + chunk_products, side="right")) - 1
        r1 = min(max(r1, r0 + 1), A.rows)
        cnt = O.symbolic(A, B, r0, r1, threads)
        counts[r0:r1] = cnt
        cp = np.zeros(r1 - r0 + 1, np.uint64)
        np.cumsum(cnt, out=cp[1:])
        n = int(cp[-1])
        if cj is None or cj.size < n:
            cj = np.empty(max(n, 1), np.uint32)
            cx = np.empty(max(n, 1), np.float64)
        ap = np.ascontiguousarray(A.rowptr, dtype=np.uint64)
        bp = np.ascontiguousarray(B.rowptr, dtype=np.uint64)
        rc = O._L().oracle_numeric(A.rows, A.nnz, O._p(ap), O._p(A.col), O._p(A.val), B.rows, B.nnz, O._p(bp),
                                   O._p(B.col), O._p(B.val), B.cols, r0, r1, O._p(cp), O._p(cj), O._p(cx), 0,
                                   threads)
        if rc:
            raise RuntimeError("oracle_numeric failed")
        r0 = r1
    return time.perf_counter() - t0, int(prod.sum()), counts


CPU_SAMPLE_PRODUCTS = 2.3e9  # products of one CPU sample (about 5 s of OpenMP Gustavson on 16 cores)


def cpu_sample_rows(A, B, threads: int):
    """The rows of the bounded CPU sample, the same for the reference arm and
    the cpu_baseline leg: every s-th row of A, s = round(products /
    CPU_SAMPLE_PRODUCTS) (all rows when the product is smaller)."""
    from oracle import oracle as O
    prod_all, _, _ = O.row_stats(A, B, threads)
    total = float(prod_all.sum())
    s = max(1, int(round(total / CPU_SAMPLE_PRODUCTS)))
    return np.arange(0, A.rows, s), s, int(total)


def cpu_sample(A, B, threads: int, repeats: int = 2):
    """The bounded CPU sample timed `repeats` times (symbolic + numeric each)."""
    rows, s, _ = cpu_sample_rows(A, B, threads)
    sub = take_rows(A, rows)
    t_all, p_all, counts = 0.0, 0, None
    for _ in range(max(1, repeats)):
        t, p, counts = cpu_gustavson(sub, B, threads)
        t_all += t
        p_all += p
    return {"seconds": t_all, "products": p_all // max(1, repeats), "stride": s, "rows": rows, "counts": counts,
            "repeats": max(1, repeats), "gflops": 2.0 * p_all / t_all / 1e9}


# ----------------------------------------------------------------------------- dist
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------------------- arms
def run_reference(args, world, rank):
    """CPU restatement of the path on the host cores (bounded samples)."""
    if rank != 0:
        return
    A, B, desc = make_workload(args.workload)
    threads = os.cpu_count() or 1
    rows, stride, total = cpu_sample_rows(A, B, threads)
    sub = take_rows(A, rows)
    cpu_gustavson(sub, B, threads)  # one untimed run: page cache and thread pool warm
    times, prods = [], []
    for _ in range(args.steps):
        t, p, _ = cpu_gustavson(sub, B, threads)
        times.append(t)
        prods.append(p)
    value = 2.0 * sum(prods) / sum(times) / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GFLOP/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "rows": A.rows, "nnz_A": A.nnz, "products": total},
        "cpu_baseline": {"value": round(value, 4), "unit": "GFLOP/s", "cores": threads, "kind": "port",
                         "sample": f"every {stride}th row of A ({rows.size} rows, {prods[0]} products "
                                   f"per step), symbolic+numeric OpenMP Gustavson (oracle/gustavson.c)"},
        "e2e": {"value": round(value, 4), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU SpGEMM; this arm times the project's CPU restatement of its "
                "algorithm on the host cores",
    }
    if not args.no_extra:
        line["reference_gpu_build"] = reference_gpu_build()
    print(json.dumps(line), flush=True)


def reference_gpu_build(names=("laplacian256", "rect")) -> dict:
    """The reference's own CUDA build (oracle/_ref/spgemm_ref, compiled from
    its sources with NUM_SM = 148 by `make -C oracle refbin`) on the Laplacian
    256^2 and the rectangular A*A^T, through its own driver with 10 warm-up and 10 timed iterations; its
    stats JSON gives its mean time per multiply. Skipped where the build or a
    GPU is missing. (The R-MAT 2^20 multiply is not run: nnz(C) exceeds the reference's
    32-bit row offsets, and a wrapped offset would write out of bounds.)"""
    import shutil
    import tempfile
    ref = ROOT / "oracle" / "_ref" / "spgemm_ref"
    if not ref.exists() or shutil.which("nvidia-smi") is None:
        return {"skipped": "reference build or GPU not present"}
    from research_b200 import matrices as M
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for name in names:
            A, B, desc = make_workload(name)
            pa = Path(td) / "a.mtxd_.hicsr"
            M.write_hicsr(A, pa)
            cmd = [str(ref), str(pa)]
            if B is not A:
                pb = Path(td) / "b.mtxd_.hicsr"
                M.write_hicsr(B, pb)
                cmd.append(str(pb))
            stats = Path(td) / "stats.json"
            cfg = Path(td) / "cfg.json"
            cfg.write_text(json.dumps({"warmup_iters": 10, "bench_iters": 10, "check_correctness": False,
                                       "output_stats": True, "stats_output_file": str(stats),
                                       "print_info": False, "track_stage_time": False}))
            cmd.append(str(cfg))
            try:
                r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
                if r.returncode != 0:
                    out[name] = {"error": f"rc={r.returncode}: {r.stderr[-300:]}"}
                    continue
                st = json.loads(stats.read_text())
                out[name] = {"workload": desc, "reference_ms": round(float(st["total_time"]), 4),
                             "reference_gflops": round(float(st["gflops"]), 3),
                             "reference_workflow": st["decision"]["workflow"], "num_sm": 148,
                             "iterations": "10 warm-up, 10 timed (config/bench.json's counts)"}
            except Exception as e:  # report, keep the line
                out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def run_ours(args, world, rank, local):
    import torch
    from research_b200.ocean import CsrOut, DeviceCSR, HostCSR, SpGEMM, _check, _ptr, lib

    torch.cuda.set_device(local)
    A, B, desc = make_workload(args.workload)
    same = B is A
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    # ---- CPU baseline first (host memory is still free), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(A, B, os.cpu_count() or 1, repeats=args.cpu_repeats)

    # ---- device-resident throughput (a handle without stage events)
    g0 = SpGEMM(dict(args.config))
    dA = DeviceCSR.from_host(A)
    dB = dA if same else DeviceCSR.from_host(B)
    for _ in range(args.warmup):
        C = g0.multiply(dA, dB, sptr)
        C.free(sptr)
    st0 = g0.get_stats()
    nnz_c = int(st0["C"]["nnz"])
    products = int(st0["stats"]["intermediate_product"])
    clocks = clock_sampler(local)
    torch.cuda.synchronize()
    barrier(world)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        C = g0.multiply(dA, dB, sptr)
        C.free(sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    elapsed = max_over_ranks(e0.elapsed_time(e1), world)
    ms = elapsed / args.steps
    value = world * 2.0 * products * args.steps / (elapsed / 1e3) / 1e9

    # ---- per-stage device times (CUDA events per class; a second handle, not in the timed region)
    g = SpGEMM({**args.config, "track_stage_time": True})
    classes = ("esc1", "esc2", "esc4", "hash_s", "hash_m", "hash_l", "bitmap")
    stage_names = ["analysis", "scan"] + [f"symbolic_{c}" for c in classes] + [f"numeric_{c}" for c in classes]
    stage_ms = {k: 0.0 for k in stage_names}
    g.multiply(dA, dB, sptr).free(sptr)
    stage_steps = max(1, min(args.steps, 3))
    for _ in range(stage_steps):
        C = g.multiply(dA, dB, sptr)
        for k in stage_names:
            stage_ms[k] += max(g.stage_ms(k), 0.0)
        C.free(sptr)
    st = g.get_stats()
    for k in stage_ms:
        stage_ms[k] /= stage_steps

    # ---- roofline of the dominant kernel
    peak, peak_kind = measured_peaks()
    dom = max(stage_ms, key=stage_ms.get)
    cls = st["classes"]
    if dom.startswith("numeric_"):
        c = cls["numeric"][dom[len("numeric_"):]]
        alg = 12 * c["nnz"] + 12 * c["a_nnz"] + 12 * B.nnz + 8 * c["rows"] + 4 * (B.rows + 1)
        alg_desc = "12 B x C entries written + 12 B x A entries of its rows + 12 B x nnz(B) + row metadata"
    elif dom.startswith("symbolic_"):
        c = cls["symbolic"][dom[len("symbolic_"):]]
        alg = 4 * c["a_nnz"] + 4 * B.nnz + 4 * (B.rows + 1) + 12 * c["rows"]
        alg_desc = "4 B x A entries of its rows + 4 B x nnz(B) + row metadata"
    else:
        alg = 16 * A.rows
        alg_desc = "row metadata"
    achieved = alg / (stage_ms[dom] / 1e3) / 1e9 if stage_ms[dom] > 0 else 0.0
    traffic = None
    tfile = ROOT / "profiles" / f"traffic_{args.workload}.json"
    if tfile.exists():
        try:
            traffic = json.loads(tfile.read_text()).get(dom)
        except Exception:
            traffic = None
    comp = compulsory_bytes(A, B, nnz_c)

    # ---- parity spot check against the oracle (rows of the CPU sample + heavy rows)
    parity = None
    if rank == 0 and not args.no_check:
        from oracle import oracle as O
        C = g.multiply(dA, dB, sptr)
        check_rows = [0, 1, 2, A.rows // 2, A.rows - 1] + list(range(3, A.rows, max(1, A.rows // 24)))[:24]
        worst = 0.0
        for r in sorted(set(check_rows)):
            rp, col, val = C.download_rows(r, r + 1)
            cp, cj, cx, ca = O.spgemm(A, B, r, r + 1, with_abs=True)
            worst = max(worst, O.compare(rp - rp[0], col, val, cp, cj, cx, ca, 1e-12))
        counts_ok = None
        if cpu is not None:
            rows = cpu["rows"]
            full = np.empty(A.rows + 1, np.uint64)
            _check(lib().ocean_csr_download_rows(ctypes.byref(C._out), 0, A.rows, _ptr(full), 0, 0, None))
            gpu_counts = full[rows + 1] - full[rows]
            counts_ok = bool(np.array_equal(gpu_counts, cpu["counts"]))
        C.free(sptr)
        parity = {"rows_checked_exact": len(set(check_rows)), "max_rel_err": worst, "tolerance": 1e-12,
                  "cpu_sample_row_counts_equal": counts_ok}

    # ---- the same product as a one-problem captured plan (ocean_batch_*): the
    # repeated-structure form, whose launches replay a CUDA graph without the
    # per-call read-backs; only where a second C fits easily beside the first
    plan_line = None
    if 12 * nnz_c < 8e9:
        from research_b200.ocean import Batch
        gb = SpGEMM({})
        plan = Batch(gb, [dA], [dB], sptr)
        for _ in range(args.warmup):
            plan.launch(sptr)
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(args.steps):
            plan.launch(sptr)
        p1.record(stream)
        torch.cuda.synchronize()
        pms = max_over_ranks(p0.elapsed_time(p1), world) / args.steps
        pinfo = plan.info()
        out = plan.run(sptr)[0]
        plan_same = int(out.nnz) == nnz_c
        plan_line = {"value": round(world * 2.0 * products / (pms / 1e3) / 1e9, 3), "ms_per_step": round(pms, 4),
                     "speedup_vs_plain": round(ms / pms, 3), "workflow": pinfo["workflow"],
                     "kernel_launches": pinfo["kernel_launches"], "nnz_C_equal": plan_same,
                     "api": "ocean_batch_create once, ocean_batch_launch per step (captured graph)"}
        plan.close()
        gb.close()

    # ---- end to end through the host-buffer C ABI (pinned inputs, host output);
    # the two device-input handles give back their workspaces and saved bitmaps first
    g0.close()
    g.close()
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, A, B, same, nnz_c, products, world, stream)

    configs = None
    if world == 1 and not args.no_extra:
        del dA, dB
        release_memory()
        configs = extra_legs(args, stream)

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "rows": A.rows, "cols": B.cols, "nnz_A": A.nnz, "nnz_B": B.nnz,
                   "products": products, "nnz_C": nnz_c, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (A is %.0f MB, C %.1f GB)" % (
                       (12 * A.nnz + 4 * A.rows) / 1e6, 12 * nnz_c / 1e9)},
        "hbm_gbs_compulsory": round(comp / (ms / 1e3) / 1e9, 2),
        "gather_gbs_effective": round(12 * products / (ms / 1e3) / 1e9, 2),
        "stage_ms": {k: round(v, 4) for k, v in stage_ms.items() if v > 0},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "algorithmic_bytes_per_launch": int(alg), "algorithmic_bytes": alg_desc,
                     "launch_ms": round(stage_ms[dom], 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
        "cpu_baseline": None if cpu is None else {
            "value": round(cpu["gflops"], 4), "unit": "GFLOP/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"every {cpu['stride']}th row of A ({cpu['rows'].size} rows, {cpu['products']} products; "
                      f"the reference arm's sample), symbolic+numeric OpenMP Gustavson, {cpu['repeats']} runs, "
                      f"{cpu['seconds']:.1f} s"},
        "e2e": e2e,
        "gpu_launches": int(st["decision"].get("kernel_launches", KERNELS_PER_MULTIPLY)) * args.steps,
        "clocks": clk,
        "parity": parity,
    }
    if plan_line is not None:
        line["captured_plan"] = plan_line
    if configs is not None:
        line["configs"] = configs
    print(json.dumps(line), flush=True)


def run_e2e(args, A, B, same, nnz_c, products, world, stream):
    import torch
    from research_b200.ocean import CsrOut, CsrView, SpGEMM, _check, lib

    need = 12 * nnz_c + 8 * (A.rows + 1) + 2 * (12 * A.nnz + 8 * A.rows) + (16 << 30)
    avail = 0
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                avail = int(line.split()[1]) * 1024
    except Exception:
        pass
    # every rank on this node pins its own copy of C: all of them must fit at
    # once, and all ranks take the same decision (the leg has collectives)
    local_world = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
    fits = not avail or avail >= need * local_world
    if world > 1:
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        flag = torch.tensor([1 if fits else 0], dtype=torch.int32, device=dev)
        dist.all_reduce(flag, op=dist.ReduceOp.MIN)
        fits = bool(flag.item())
    if not fits:
        return {"value": None, "unit": "GFLOP/s",
                "note": f"skipped: host has {avail / 2**30:.0f} GiB available, {local_world} rank(s) need "
                        f"{need * local_world / 2**30:.0f} GiB of pinned memory"}

    def pinned(a: np.ndarray) -> np.ndarray:
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype)[: a.size]
        v[:] = a
        pinned.keep.append(t)
        return v
    pinned.keep = []

    def pin_csr(m):
        from research_b200.ocean import HostCSR
        return HostCSR(m.rows, m.cols, pinned(m.rowptr), pinned(m.col), pinned(m.val))

    pA = pin_csr(A)
    pB = pA if same else pin_csr(B)
    g = SpGEMM(dict(args.config))
    av, bv = pA.view(), pB.view()
    out = CsrOut()
    sptr = stream.cuda_stream
    for _ in range(max(1, min(args.warmup, 2))):  # the first call also pins the host output buffers
        _check(lib().ocean_spgemm_host(g._h, ctypes.byref(av), ctypes.byref(bv), ctypes.byref(out), sptr))
    steps = args.e2e_steps or args.steps
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        _check(lib().ocean_spgemm_host(g._h, ctypes.byref(av), ctypes.byref(bv), ctypes.byref(out), sptr))
    e1.record(stream)
    torch.cuda.synchronize()
    elapsed = max_over_ranks(e0.elapsed_time(e1), world)
    h2d = A.rowptr.nbytes + A.col.nbytes + A.val.nbytes + (0 if same else B.rowptr.nbytes + B.col.nbytes + B.val.nbytes)
    d2h = (out.rows + 1) * (out.rowptr_bits // 8) + 12 * out.nnz
    chunks = int(g.get_stats().get("decision", {}).get("host_pipeline_chunks", 0))
    g.close()
    return {"value": round(world * 2.0 * products * steps / (elapsed / 1e3) / 1e9, 3), "unit": "GFLOP/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": steps,
            "ms_per_step": round(elapsed / steps, 3), "host_pipeline_chunks": chunks,
            "api": "ocean_spgemm_host (pinned host A/B in, C copied back to pinned host buffers; numeric phase "
                   "in row chunks whose copies overlap the later chunks when host_pipeline_chunks > 0)"}


# ----------------------------------------------------------------------------- further workloads
# The default run also measures the metric's other forms on one GPU, each with
# its own fixed, small step counts so the whole run stays within minutes:
# the Laplacian 256^2 and the rectangular A*A^T as plain calls, as a
# one-problem captured plan and end to end; learned row sizing of the
# held-out R-MAT 2^21 against HLL and exact counts; 512 products (learned +
# batched against 512 plain calls, with the HLL- and
# exact-sized batched forms beside it, on the device and end to end).

def _ev():
    import torch
    return torch.cuda.Event(enable_timing=True)


def time_on_device(fn, steps: int, warmup: int, stream, reps: int = 1) -> float:
    """Mean ms per call of fn() over `steps` calls after `warmup`, CUDA events on
    `stream`; with reps > 1 the median of that many such means (the forms that
    read counters back to the host between their launches are exposed to host
    scheduling stalls, which a median of repeated means does not carry)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    means = []
    for _ in range(max(1, reps)):
        e0, e1 = _ev(), _ev()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        means.append(e0.elapsed_time(e1) / steps)
    return float(np.median(means))


def leg_small(name: str, stream, steps: int = 20, warmup: int = 5, check: bool = True) -> dict:
    import torch
    from research_b200.ocean import Batch, CsrOut, DeviceCSR, SpGEMM, _check, lib
    A, B, desc = make_workload(name)
    same = B is A
    sptr = stream.cuda_stream
    dA = DeviceCSR.from_host(A)
    dB = dA if same else DeviceCSR.from_host(B)
    g = SpGEMM({})
    plain_ms = time_on_device(lambda: g.multiply(dA, dB, sptr).free(sptr), steps, warmup, stream, reps=5)
    st = g.get_stats()
    products, nnz_c = int(st["stats"]["intermediate_product"]), int(st["C"]["nnz"])
    out = {"workload": desc, "products": products, "nnz_C": nnz_c, "workflow": st["decision"]["workflow"],
           "plain_ms": round(plain_ms, 4), "plain_gflops": round(2.0 * products / plain_ms / 1e6, 3),
           "kernel_launches": st["decision"]["kernel_launches"],
           "timing": f"median of 5 means of {steps} calls each (CUDA events on the launching stream)"}
    if check:
        from oracle import oracle as O
        C = g.multiply(dA, dB, sptr)
        h = C.download()
        C.free(sptr)
        cp, cj, cx, ca = O.spgemm(A, B, with_abs=True)
        out["parity_max_rel_err"] = O.compare(h.rowptr, h.col, h.val, cp, cj, cx, ca, 1e-12)
    gb = SpGEMM({})
    plan = Batch(gb, [dA], [dB], sptr)
    plan_ms = time_on_device(lambda: plan.launch(sptr), steps, warmup, stream, reps=5)
    out["captured_plan_ms"] = round(plan_ms, 4)
    out["captured_plan_launches"] = plan.info()["kernel_launches"]
    plan.close()
    gb.close()
    # end to end: pinned host inputs, C copied back (ocean_spgemm_host)
    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype)[: a.size]
        v[:] = a
        pinned.keep.append(t)
        return v
    pinned.keep = []
    from research_b200.ocean import HostCSR
    pA = HostCSR(A.rows, A.cols, pinned(A.rowptr), pinned(A.col), pinned(A.val))
    pB = pA if same else HostCSR(B.rows, B.cols, pinned(B.rowptr), pinned(B.col), pinned(B.val))
    av, bv = pA.view(), pB.view()
    res = CsrOut()
    e2e_ms = time_on_device(lambda: _check(lib().ocean_spgemm_host(g._h, ctypes.byref(av), ctypes.byref(bv),
                                                                   ctypes.byref(res), sptr)),
                            steps, warmup, stream, reps=5)
    out["e2e_ms"] = round(e2e_ms, 4)
    out["e2e_gflops"] = round(2.0 * products / e2e_ms / 1e6, 3)
    g.close()
    # CPU baseline of the whole product (OpenMP Gustavson, all host cores; median of 5)
    threads = os.cpu_count() or 1
    cpu_gustavson(A, B, threads)
    ts = sorted(cpu_gustavson(A, B, threads)[0] for _ in range(5))
    out["cpu_ms"] = round(1e3 * ts[2], 3)
    out["cpu_gflops"] = round(2.0 * products / ts[2] / 1e9, 3)
    out["cpu_cores"] = threads
    return out


def leg_sizing(stream, steps: int = 3, warmup: int = 2) -> dict:
    """Row sizes of C = A*A for the held-out R-MAT n = 2^21 (24 per
    row, seed 7; generated on the device; C, ~0.55 TB, is never formed) by
    exact symbolic counts, HLL and the learned network, with the estimates'
    errors against the exact counts on the rows they size (> 128 products)."""
    import torch
    from research_b200 import estimator as E
    from research_b200.ocean import SpGEMM
    A = E.generate("rmat", 1 << 21, 24, seed=7)
    g = SpGEMM({})
    truth = g.symbolic(A, A)
    exact_ms = time_on_device(lambda: g.symbolic(A, A), steps, warmup, stream)
    res = {}
    for name in ("learned", "hll"):
        ms = time_on_device(lambda: E.estimate(g, A, None, name, True), steps, warmup, stream)
        est = E.estimate(g, A, None, name, True)
        raw = E.estimate(g, A, None, name, False)
        res[name] = {"ms": round(ms, 3), "prealloc": E.metrics(g, est, truth, 128), "raw": E.metrics(g, raw, truth, 128)}
    g.close()
    return {"workload": "R-MAT n=2^21, 24 entries/row, seed 7 (held out from training); row sizes of C=A*A",
            "rows": A.rows, "nnz_A": A.nnz, "exact_symbolic_ms": round(exact_ms, 3), "learned": res["learned"],
            "hll": res["hll"], "speedup_learned_vs_exact": round(exact_ms / res["learned"]["ms"], 2),
            "speedup_learned_vs_hll": round(res["hll"]["ms"] / res["learned"]["ms"], 3)}


def leg_batch(stream, steps: int = 3, warmup: int = 2, e2e_steps: int = 2, ablation: bool = True,
              check: bool = True) -> dict:
    """512 independent A_p*A_p (n log-uniform 1k-64k; banded, R-MAT,
    uniform and block-diagonal in turn; 4-32 entries per row; FP64; generated
    on the device, seed 5). Plain: 512 sequential ocean_spgemm calls. Learned +
    batched: one captured graph of the whole batch, rows sized by the network,
    class policy autotuned. Ablation: the same batched graph sized by HLL, and
    by exact symbolic counts. End to end: pinned host inputs copied in, every
    result copied back (batched: ocean_batch_download; plain: 512
    ocean_spgemm_host calls)."""
    import torch
    from research_b200 import estimator as E
    from research_b200.ocean import Batch, CsrOut, HostCSR, SpGEMM, _check, lib
    sptr = stream.cuda_stream
    specs = E.training_specs(512, seed=5, n_lo=1024, n_hi=65536)
    dA = [E.generate(sp.kind, sp.n, sp.deg, sp.seed, sp.param) for sp in specs]
    torch.cuda.synchronize()
    gp = SpGEMM({})
    products = 0
    for a in dA:
        C = gp.multiply(a, a, sptr)
        products += int(gp.get_stats()["stats"]["intermediate_product"])
        C.free(sptr)

    def plain_step():
        for a in dA:
            gp.multiply(a, a, sptr).free(sptr)
    plain_ms = time_on_device(plain_step, 1, warmup, stream, reps=max(3, steps))
    gf = lambda ms: round(2.0 * products / (ms / 1e3) / 1e9, 3)
    out = {"workload": "512 x A_p*A_p, n log-uniform 1k-64k, banded/R-MAT/uniform/block-diagonal in turn, "
                       "4-32 entries per row, FP64 U[-1,1], seed 5", "products": products,
           "plain": {"ms": round(plain_ms, 3), "gflops": gf(plain_ms),
                     "form": f"512 sequential ocean_spgemm calls; median of {max(3, steps)} such steps"}}

    def batched(config):
        gb = SpGEMM(config)
        t0 = time.time()
        plan = Batch(gb, dA, stream=sptr)
        plan_s = time.time() - t0
        ms = time_on_device(lambda: plan.launch(sptr), steps, warmup, stream)
        return gb, plan, ms, plan_s

    forms = [("learned_batched", {"use_learned_estimator": True, "batch_autotune": True})]
    if ablation:
        forms += [("hll_batched", {"force_workflow": 1}), ("exact_batched", {"force_workflow": 0})]
    for name, cfg in forms:
        gb, plan, ms, plan_s = batched(cfg)
        info = plan.info()
        rec = {"ms": round(ms, 3), "gflops": gf(ms), "speedup_vs_plain": round(plain_ms / ms, 3),
               "plan_seconds": round(plan_s, 2), "kernel_launches": info["kernel_launches"],
               "workflow": info["workflow"], "estimator": info.get("estimator"), "nnz_C": int(info["nnz_c"])}
        if name == "learned_batched":
            rec["tuning"] = info.get("tuning")
            res = plan.run(sptr)
            if check:
                from oracle import oracle as O
                worst = 0.0
                for q in range(0, 512, 37):
                    h = res[q].download()
                    A = dA[q].download()
                    rp, cj, cx, ca = O.spgemm(A, A, with_abs=True)
                    worst = max(worst, O.compare(h.rowptr, h.col, h.val, rp, cj, cx, ca, 1e-12))
                rec["parity"] = {"problems_checked": len(range(0, 512, 37)), "max_rel_err": worst}
            if e2e_steps > 0:
                hosts = [(pinned_like(a.rowptr), pinned_like(a.col), pinned_like(a.val)) for a in dA]
                nnz_c = int(info["nnz_c"])
                wide = info["rowptr_bits"] == 64
                outs = (torch.empty(int(info["rows"]) + len(dA), dtype=torch.int64 if wide else torch.int32,
                                    pin_memory=True),
                        torch.empty(max(nnz_c, 1), dtype=torch.int32, pin_memory=True),
                        torch.empty(max(nnz_c, 1), dtype=torch.float64, pin_memory=True))
                rec["e2e"] = batch_e2e(plan, info, dA, gp, stream, e2e_steps, hosts, outs)
                out["plain"]["e2e_ms"] = rec["e2e"].pop("plain_ms")
                out["plain"]["e2e_gflops"] = gf(out["plain"]["e2e_ms"])
                rec["e2e"]["gflops"] = gf(rec["e2e"]["ms"])
                rec["e2e_speedup_vs_plain"] = round(out["plain"]["e2e_ms"] / rec["e2e"]["ms"], 3)
        out[name] = rec
        plan.close()
        gb.close()
        if name == "learned_batched" and e2e_steps > 0:
            # the same batch as 8 plans of 64 problems with the tuned policy,
            # pipelined over three streams: inputs of plan i+1 copied in and
            # plan i computed while plan i-1's results are copied back
            tuned = {k: info[k] for k in ("esc_max_products", "hash_s_max_scale", "bitmap_words_scale") if k in info}
            pe = batch_e2e_pipelined(dA, {"use_learned_estimator": True, **tuned}, stream, e2e_steps, hosts, outs,
                                     chunks=8)
            del hosts, outs
            pe["gflops"] = gf(pe["ms"])
            rec["e2e_pipelined"] = pe
            rec["e2e_pipelined_speedup_vs_plain"] = round(out["plain"]["e2e_ms"] / pe["ms"], 3)
    gp.close()
    return out


def pinned_like(t):
    import torch
    return torch.empty(t.shape, dtype=t.dtype, pin_memory=True).copy_(t.cpu())


def batch_e2e(plan, info, dA, gp, stream, steps: int, hosts, outs) -> dict:
    """End-to-end ms of one batched step and of 512 plain host-buffer calls
    (hosts: pinned copies of the inputs; outs: pinned rowptr, col, val arrays)."""
    import torch
    from research_b200.ocean import CsrOut, HostCSR, _check, lib
    sptr = stream.cuda_stream
    nnz_c = int(info["nnz_c"])
    rp_out, col_out, val_out = outs

    def step():
        for a, (r, c, v) in zip(dA, hosts):
            a.rowptr.copy_(r, non_blocking=True)
            a.col.copy_(c, non_blocking=True)
            a.val.copy_(v, non_blocking=True)
        plan.launch(sptr)
        plan.download_into(rp_out.numpy(), col_out.numpy(), val_out.numpy(), sptr)
    ms = time_on_device(step, steps, 1, stream)
    hcsr = [HostCSR(a.rows, a.cols, r.numpy().view(np.uint32) if a.rowptr_bits == 32 else r.numpy().view(np.uint64),
                    c.numpy().view(np.uint32), v.numpy()) for a, (r, c, v) in zip(dA, hosts)]
    res = CsrOut()

    def plain():
        for m in hcsr:
            mv = m.view()
            _check(lib().ocean_spgemm_host(gp._h, ctypes.byref(mv), ctypes.byref(mv), ctypes.byref(res), sptr))
    plain_ms = time_on_device(plain, steps, 1, stream)
    return {"ms": round(ms, 3), "plain_ms": round(plain_ms, 3),
            "h2d_bytes_per_step": int(sum(x.nbytes for hs in hosts for x in hs)),
            "d2h_bytes_per_step": int(rp_out.nbytes + 12 * nnz_c),
            "api": "pinned host inputs -> device, ocean_batch_launch, ocean_batch_download; "
                   "plain: 512 x ocean_spgemm_host"}


def batch_e2e_pipelined(dA, config: dict, stream, steps: int, hosts, outs, chunks: int = 8) -> dict:
    """End-to-end ms of one step of the batch as `chunks` captured plans on
    three streams (copy in, compute, copy out; ocean_batch_launch and
    ocean_batch_download_async), CUDA events on `stream` around the step."""
    import torch
    from research_b200.ocean import Batch, SpGEMM
    n = len(dA)
    bounds = [round(i * n / chunks) for i in range(chunks + 1)]
    g = SpGEMM(config)
    plans, parts = [], []
    for i in range(chunks):
        part = dA[bounds[i]:bounds[i + 1]]
        plans.append(Batch(g, part, stream=stream.cuda_stream))
        parts.append(part)
    infos = [pl.info() for pl in plans]
    # each plan's inputs are slices of the pinned input copies; its results go
    # to consecutive slices of the shared pinned outputs (row pointers as
    # 64-bit words, enough for either width)
    chunk_hosts = [hosts[bounds[i]:bounds[i + 1]] for i in range(chunks)]
    rp_all, col_all, val_all = outs
    rp64 = rp_all.view(torch.int64) if rp_all.dtype == torch.int64 else None
    chunk_outs, e_at, r_at = [], 0, 0
    for inf in infos:
        nnz, nr = int(inf["nnz_c"]), int(inf["rows"]) + int(inf["problems"])
        rp_view = (torch.empty(nr, dtype=torch.int64 if inf["rowptr_bits"] == 64 else torch.int32, pin_memory=True)
                   if rp64 is None or inf["rowptr_bits"] != 64 else rp64[r_at:r_at + nr])
        chunk_outs.append((rp_view, col_all[e_at:e_at + max(nnz, 1)], val_all[e_at:e_at + max(nnz, 1)]))
        e_at += nnz
        r_at += nr
    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()

    def step():
        start = torch.cuda.Event()
        start.record(stream)
        for st in (s_in, s_comp, s_out):
            st.wait_event(start)
        done = None
        for pl, part, hs, (rp, col, val) in zip(plans, parts, chunk_hosts, chunk_outs):
            with torch.cuda.stream(s_in):
                for a, (r, c, v) in zip(part, hs):
                    a.rowptr.copy_(r, non_blocking=True)
                    a.col.copy_(c, non_blocking=True)
                    a.val.copy_(v, non_blocking=True)
            e_in = torch.cuda.Event()
            e_in.record(s_in)
            s_comp.wait_event(e_in)
            pl.launch(s_comp.cuda_stream)
            e_c = torch.cuda.Event()
            e_c.record(s_comp)
            s_out.wait_event(e_c)
            pl.download_into(rp.numpy(), col.numpy(), val.numpy(), s_out.cuda_stream, wait=False)
            done = torch.cuda.Event()
            done.record(s_out)
        stream.wait_event(done)
    ms = time_on_device(step, steps, 1, stream)
    res = {"ms": round(ms, 3), "chunks": chunks, "kernel_launches_per_plan": infos[0]["kernel_launches"],
           "h2d_bytes_per_step": int(sum(x.nbytes for h in hosts for x in h)),
           "d2h_bytes_per_step": int(sum(o[0].nbytes + 12 * int(inf["nnz_c"]) for o, inf in zip(chunk_outs, infos))),
           "api": "8 x (ocean_batch_create once; per step ocean_batch_launch, ocean_batch_download_async) "
                  "on copy-in/compute/copy-out streams"}
    for pl in plans:
        pl.close()
    g.close()
    return res


def extra_legs(args, stream) -> dict:
    out = {}
    for name, fn in (("laplacian256", lambda: leg_small("laplacian256", stream, check=not args.no_check)),
                     ("rect", lambda: leg_small("rect", stream, check=not args.no_check)),
                     ("rmat21_sizing", lambda: leg_sizing(stream)),
                     ("batch512", lambda: leg_batch(stream, check=not args.no_check,
                                                     e2e_steps=0 if args.no_e2e else 2))):
        t0 = time.time()
        try:
            out[name] = fn()
        except Exception as e:  # report, keep the headline line
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["leg_seconds"] = round(time.time() - t0, 1)
        release_memory()
    return out


def release_memory():
    """Returns cached device memory and torch's cached pinned host buffers
    (a leg pins up to ~120 GB of host memory for its copies)."""
    import gc
    import torch
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    if hasattr(torch._C, "_host_emptyCache"):
        torch._C._host_emptyCache()



def run_batch(args, world, rank, local):
    """Workload batch512 alone: see leg_batch."""
    import torch
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    clocks = clock_sampler(local)
    clocks.start()
    r = leg_batch(stream, steps=args.steps, warmup=args.warmup, e2e_steps=0 if args.no_e2e else args.e2e_steps,
                  check=not args.no_check)
    clk = clocks.stop()
    lb = r["learned_batched"]
    line = {"metric": METRIC + " (batch of 512 independent products)", "value": lb["gflops"], "unit": "GFLOP/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": lb["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batch512: " + r["workload"], "products": r["products"]},
            "e2e": None if "e2e" not in lb else {"value": lb["e2e"]["gflops"], "unit": "GFLOP/s",
                                                 "h2d_bytes_per_step": lb["e2e"]["h2d_bytes_per_step"],
                                                 "d2h_bytes_per_step": lb["e2e"]["d2h_bytes_per_step"]},
            "gpu_launches": int(lb["kernel_launches"]) * args.steps, "clocks": clk, "batch512": r}
    print(json.dumps(line), flush=True)


def run_sizing(args, world, rank, local):
    """Workload rmat21-sizing alone: see leg_sizing."""
    import torch
    torch.cuda.set_device(local)
    r = leg_sizing(torch.cuda.current_stream(), steps=args.steps, warmup=args.warmup)
    r["steps"], r["warmup"] = args.steps, args.warmup
    print(json.dumps(r), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat20")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-repeats", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="headline workload only (no configs 1, 3, 4, 5)")
    ap.add_argument("--config", type=json.loads, default={},
                    help="library configuration (JSON object) for the headline workload's handles, e.g. "
                         "'{\"numeric_windows\": true}' when profiling a kernel variant")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("note: fewer than 3 warm-up steps", file=sys.stderr)
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "batch512":
            run_batch(args, world, rank, local)
        elif args.workload == "rmat21-sizing":
            run_sizing(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
