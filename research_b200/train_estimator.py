"""Trains the learned row-size estimator on the GPU and writes its weights.

    python -m research_b200.train_estimator [--matrices 2000] [--steps 6000]
        [--out research_b200/estimator_weights.txt] [--inc research_b200/csrc/mlp_weights.inc]
        [--eval-scale 21 --eval-deg 24] [--report report.json]

Training set: seeded A*A products over four families (banded with bandwidth
3-65, R-MAT, uniform random, block-diagonal with 32-256-wide blocks), 4-32
entries per row: `--matrices` products with n log-uniform in 16k-1M and
`--small-matrices` more with n log-uniform in 1k-64k (the sizes of batched
workloads); every row with more than 128 products is a candidate (at most 4096
per product), labelled with its exact output count from the library's
symbolic pass. One product in ten is held out
for validation and for the safety margin (the 98th percentile of the
under-prediction). Forward and backward passes are the library's tensor-core
kernels; the optimiser is the library's Adam kernel.

Evaluation: a held-out R-MAT (2^eval-scale rows, eval-deg entries per row)
whose exact counts come from the symbolic pass (its C is never formed); the
learned estimates and the HLL estimates of the reference's workflow are scored
on the rows they size (more than 128 products): mean relative row-size error,
share of rows whose numeric class is wrong, rows below the truth (reruns) and
total preallocated slots.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import estimator as E
from .ocean import MLP_BLOB, SpGEMM

HERE = Path(__file__).resolve().parent


def write_inc(path: Path, blob: np.ndarray, note: str) -> None:
    lines = ["// Built-in network of the learned row-size estimator: kMlpParams parameters,",
             "// then the 16 feature means, the 16 inverse standard deviations and the log2",
             "// margin. Written by research_b200/train_estimator.py.",
             "// " + note,
             "static const int kMlpBuiltinTrained = 1;",
             f"static const float kMlpBuiltin[{MLP_BLOB}] = {{"]
    for i in range(0, blob.size, 6):
        lines.append("    " + ", ".join("%.9ef" % x for x in blob[i:i + 6]) + ",")
    lines.append("};")
    path.write_text("\n".join(lines) + "\n")


def evaluate(g: SpGEMM, net_loaded: bool, scale: int, deg: int, seed: int, min_products: int = 128) -> dict:
    import torch
    A = E.generate("rmat", 1 << scale, deg, seed)
    t0 = time.time()
    truth = g.symbolic(A, A)
    torch.cuda.synchronize()
    out = {"matrix": f"rmat scale {scale}, {deg} per row", "rows": A.rows, "nnz": A.nnz,
           "symbolic_s": time.time() - t0}
    for name in (["learned"] if net_loaded else []) + ["hll"]:
        for margin in (False, True):
            est = E.estimate(g, A, None, name, margin)
            m = E.metrics(g, est, truth, min_products)
            m["est_total"] = int((est.to(torch.int64) & 0xFFFFFFFF).sum().item())
            out[f"{name}{'_prealloc' if margin else '_raw'}"] = m
    out["truth_total"] = int((truth.to(torch.int64) & 0xFFFFFFFF).sum().item())
    return out


def evaluate_small(g: SpGEMM, count: int, seed: int, min_products: int = 128) -> dict:
    """Held-out products of the batched sizes (n 1k-64k): totals of the
    preallocations against the exact total, rows below the truth, and the
    row-weighted mean relative error of the raw estimates."""
    import torch
    tot = {"truth": 0, "learned": 0, "hll": 0, "learned_under": 0, "hll_under": 0, "rows": 0,
           "learned_raw_err": 0.0, "hll_raw_err": 0.0}
    for sp in E.training_specs(count, seed, n_lo=1024, n_hi=65536):
        A = E.generate(sp.kind, sp.n, sp.deg, sp.seed, sp.param)
        truth = g.symbolic(A, A)
        tot["truth"] += int((truth.to(torch.int64) & 0xFFFFFFFF).sum().item())
        for name in ("learned", "hll"):
            est = E.estimate(g, A, None, name, True)
            m = E.metrics(g, est, truth, min_products)
            tot[name] += int((est.to(torch.int64) & 0xFFFFFFFF).sum().item())
            tot[name + "_under"] += m["under_rows"]
            raw = E.metrics(g, E.estimate(g, A, None, name, False), truth, min_products)
            tot[name + "_raw_err"] += raw["mean_rel_error"] * raw["rows"]
        tot["rows"] += m["rows"]
    for name in ("learned", "hll"):
        tot[name + "_raw_err"] = tot[name + "_raw_err"] / max(tot["rows"], 1)
    tot["problems"] = count
    return tot


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--matrices", type=int, default=2000)
    ap.add_argument("--small-matrices", type=int, default=1000)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--rows-per-matrix", type=int, default=4096)
    ap.add_argument("--quantile", type=float, default=0.98)
    ap.add_argument("--out", default=str(HERE / "estimator_weights.txt"))
    ap.add_argument("--inc", default="")
    ap.add_argument("--eval-scale", type=int, default=21)
    ap.add_argument("--eval-deg", type=int, default=24)
    ap.add_argument("--report", default="")
    a = ap.parse_args(argv)
    import torch
    g = SpGEMM({})
    specs = E.training_specs(a.matrices, a.seed)
    if a.small_matrices:
        specs += E.training_specs(a.small_matrices, a.seed + 1, n_lo=1024, n_hi=65536)
    val = specs[::10]
    train = [s for i, s in enumerate(specs) if i % 10]
    t0 = time.time()
    feat, target = E.dataset(g, train, a.rows_per_matrix, seed=a.seed)
    vfeat, vtarget = E.dataset(g, val, a.rows_per_matrix, seed=a.seed + 1)
    t_data = time.time() - t0
    mu, isd = E.normalisation(feat)
    net = E.Network.initial(mu, isd, seed=a.seed)
    t0 = time.time()
    losses = E.train(g, net, feat, target, a.steps, a.batch, a.lr, seed=a.seed)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    vpred = net.forward(g, vfeat)
    vloss = float(((vpred - vtarget) ** 2).mean().item())
    margin = E.calibrate_margin(g, net, vfeat, vtarget, a.quantile)
    net.save(a.out)
    report = {"train_rows": int(feat.shape[0]), "val_rows": int(vfeat.shape[0]), "matrices": a.matrices,
              "small_matrices": a.small_matrices,
              "data_s": t_data, "train_s": t_train, "steps": a.steps, "batch": a.batch,
              "loss_first": losses[0] if losses else None, "loss_last": losses[-1] if losses else None,
              "val_mse_log2": vloss, "margin_log2": margin}
    if a.inc:
        write_inc(Path(a.inc), net.blob(),
                  f"{a.matrices} + {a.small_matrices} products, {int(feat.shape[0])} training rows, {a.steps} steps of "
                  f"{a.batch}; validation MSE {vloss:.4f} (log2 units), margin {margin:.4f}")
    if a.eval_scale:
        g2 = SpGEMM({"learned_estimator_weights": str(a.out)})
        report["eval"] = evaluate(g2, True, a.eval_scale, a.eval_deg, seed=a.seed + 7)
        report["eval_small"] = evaluate_small(g2, 64, seed=a.seed + 11)
    text = json.dumps(report, indent=1)
    print(text)
    if a.report:
        Path(a.report).write_text(text)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
