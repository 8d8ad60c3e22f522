"""Host side of the learned row-size estimator.

The network (16 features -> 64 -> 64 -> 1, ReLU; BF16 weights on the tensor
cores, FP32 accumulation) predicts t = log2(1 + nnz of an output row). Its
forward and backward passes are the library's kernels (``ocean_mlp_forward``,
``ocean_mlp_grad``, ``ocean_mlp_adam``); this module keeps the parameters in
device memory (torch tensors as plumbing), draws training batches, and reads
and writes weight files (text: the tag ``ocean-mlp-v1`` then
``OCEAN_MLP_BLOB`` numbers: parameters, feature means, inverse deviations,
log2 margin).

It also generates, on the device, the seeded synthetic families the network is
trained and evaluated on: banded, R-MAT, uniform random and block-diagonal
matrices with n rows and about ``deg`` entries per row.

The reference has no learned estimator; its row sizes come from HLL
(kernels/HLL.cuh:107-236).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from .ocean import (MLP_BLOB, MLP_FEATURES, MLP_PARAMS, CsrView, DeviceCSR, MlpModel, SpGEMM, _check, _ptr, lib)

H = 64
OFF_W1, OFF_B1 = 0, H * MLP_FEATURES
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
TAG = "ocean-mlp-v1"


class Network:
    """Parameters (FP32 master copy), feature normalisation and margin, on the device."""

    def __init__(self, params, mu, inv_sd, margin: float = 0.0):
        import torch
        self.params = torch.as_tensor(np.asarray(params, np.float32)).cuda().contiguous()
        self.mu = torch.as_tensor(np.asarray(mu, np.float32)).cuda().contiguous()
        self.inv_sd = torch.as_tensor(np.asarray(inv_sd, np.float32)).cuda().contiguous()
        self.margin = float(margin)
        assert self.params.numel() == MLP_PARAMS and self.mu.numel() == MLP_FEATURES

    @staticmethod
    def initial(mu, inv_sd, seed: int = 0) -> "Network":
        """He-normal weights, zero biases."""
        rng = np.random.default_rng(seed)
        p = np.zeros(MLP_PARAMS, np.float32)
        p[OFF_W1:OFF_B1] = rng.normal(0, math.sqrt(2.0 / MLP_FEATURES), H * MLP_FEATURES)
        p[OFF_W2:OFF_B2] = rng.normal(0, math.sqrt(2.0 / H), H * H)
        p[OFF_W3:OFF_B3] = rng.normal(0, math.sqrt(1.0 / H), H)
        return Network(p, mu, inv_sd)

    @staticmethod
    def from_blob(blob) -> "Network":
        b = np.asarray(blob, np.float32)
        assert b.size == MLP_BLOB
        P, F = MLP_PARAMS, MLP_FEATURES
        return Network(b[:P], b[P:P + F], b[P + F:P + 2 * F], float(b[P + 2 * F]))

    @staticmethod
    def builtin() -> "Network":
        blob = np.empty(MLP_BLOB, np.float32)
        _check(lib().ocean_mlp_builtin(blob.ctypes.data, MLP_BLOB))
        return Network.from_blob(blob)

    @staticmethod
    def load(path) -> "Network":
        with open(path) as f:
            tok = f.read().split()
        if not tok or tok[0] != TAG or len(tok) != MLP_BLOB + 1:
            raise ValueError(f"{path}: not an {TAG} file with {MLP_BLOB} numbers")
        return Network.from_blob(np.array([float(x) for x in tok[1:]], np.float32))

    def blob(self) -> np.ndarray:
        return np.concatenate([self.params.cpu().numpy(), self.mu.cpu().numpy(), self.inv_sd.cpu().numpy(),
                               np.array([self.margin], np.float32)]).astype(np.float32)

    def save(self, path) -> None:
        b = self.blob()
        with open(path, "w") as f:
            f.write(TAG + "\n")
            for i in range(0, b.size, 8):
                f.write(" ".join("%.9g" % x for x in b[i:i + 8]) + "\n")

    def model(self, margin: Optional[float] = None) -> MlpModel:
        return MlpModel(_ptr(self.params), _ptr(self.mu), _ptr(self.inv_sd),
                        self.margin if margin is None else margin)

    def forward(self, g: SpGEMM, feat):
        """Predicted log2(1 + nnz) for feat[n][16] (device float32)."""
        import torch
        feat = feat.contiguous()
        pred = torch.empty(feat.shape[0], dtype=torch.float32, device="cuda")
        m = self.model()
        _check(lib().ocean_mlp_forward(g._h, ctypes.byref(m), _ptr(feat), feat.shape[0], _ptr(pred), None))
        return pred

    def grad(self, g: SpGEMM, feat, target, batch: float, grad_buf, loss_buf) -> None:
        """Adds d(sum (pred - target)^2 / batch)/dparams to grad_buf and the
        summed squared error to loss_buf[0]."""
        m = self.model()
        _check(lib().ocean_mlp_grad(g._h, ctypes.byref(m), _ptr(feat), _ptr(target), feat.shape[0], float(batch),
                                    _ptr(grad_buf), _ptr(loss_buf), None))


def features(g: SpGEMM, A: DeviceCSR, B: Optional[DeviceCSR] = None):
    """Raw features of every row of A*B (device float32 [rows][16])."""
    import torch
    B = A if B is None else B
    feat = torch.empty((A.rows, MLP_FEATURES), dtype=torch.float32, device="cuda")
    av, bv = A.view(), B.view()
    _check(lib().ocean_mlp_features(g._h, ctypes.byref(av), ctypes.byref(bv), _ptr(feat), None))
    return feat


def normalisation(feat) -> Tuple[np.ndarray, np.ndarray]:
    """Per-feature mean and inverse standard deviation (constant features: 1)."""
    f = feat.double()
    mu = f.mean(0).cpu().numpy()
    sd = f.std(0).cpu().numpy()
    inv = np.where(sd > 1e-6, 1.0 / np.maximum(sd, 1e-6), 1.0)
    return mu.astype(np.float32), inv.astype(np.float32)


def train(g: SpGEMM, net: Network, feat, target, steps: int, batch: int = 8192, lr: float = 2e-3,
          seed: int = 0, log_every: int = 100) -> List[float]:
    """Adam on the mean squared log2 error with cosine learning-rate decay;
    returns the mean batch loss every log_every steps."""
    import torch
    n = feat.shape[0]
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    m1 = torch.zeros(MLP_PARAMS, dtype=torch.float32, device="cuda")
    m2 = torch.zeros_like(m1)
    gbuf = torch.zeros_like(m1)
    lbuf = torch.zeros(1, dtype=torch.float32, device="cuda")
    losses, acc = [], 0.0
    for step in range(1, steps + 1):
        idx = torch.randint(0, n, (batch,), generator=gen, device="cuda")
        f = feat.index_select(0, idx).contiguous()
        t = target.index_select(0, idx).contiguous()
        lbuf.zero_()
        net.grad(g, f, t, batch, gbuf, lbuf)
        lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * (step - 1) / steps))
        _check(lib().ocean_mlp_adam(g._h, _ptr(net.params), _ptr(m1), _ptr(m2), _ptr(gbuf), step, lr_t, 0.9, 0.999,
                                    1e-8, None))
        acc += float(lbuf.item()) / batch
        if step % log_every == 0:
            losses.append(acc / log_every)
            acc = 0.0
    return losses


def calibrate_margin(g: SpGEMM, net: Network, feat, target, quantile: float = 0.98) -> float:
    """log2 margin such that `quantile` of the rows' true t is at most the
    prediction plus the margin."""
    import torch
    pred = net.forward(g, feat)
    resid = (target - pred).float()
    q = float(torch.quantile(resid[:min(resid.numel(), 1 << 24)], quantile).item())
    net.margin = max(q, 0.0)
    return net.margin


def estimate(g: SpGEMM, A: DeviceCSR, B: Optional[DeviceCSR], estimator: str, with_margin: bool):
    """Per-row estimates as the estimation workflow makes them (uint32 as int32 tensor)."""
    import torch
    B = A if B is None else B
    out = torch.empty(A.rows, dtype=torch.int32, device="cuda")
    av, bv = A.view(), B.view()
    _check(lib().ocean_estimate(g._h, ctypes.byref(av), ctypes.byref(bv), 2 if estimator == "learned" else 1,
                                1 if with_margin else 0, _ptr(out), None))
    return out


def metrics(g: SpGEMM, est, truth, min_products: int = 0) -> dict:
    """Quality of est against exact counts for the handle's last analysed A*B."""
    out = np.zeros(4, np.float64)
    _check(lib().ocean_estimate_metrics(g._h, _ptr(est), _ptr(truth), min_products, out.ctypes.data, None))
    return {"mean_rel_error": float(out[0]), "misbinned_pct": float(out[1]), "rows": int(out[2]),
            "under_rows": int(out[3])}


# ---------------------------------------------------------------- families

FAMILIES = ("banded", "rmat", "uniform", "block")


def _csr(n: int, cols: int, r, c, gen) -> DeviceCSR:
    import torch
    key = torch.unique(r * cols + c)  # sorted, duplicates merged
    r = key // cols
    c = key - r * cols
    counts = torch.bincount(r, minlength=n)
    rowptr = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    rowptr[1:] = torch.cumsum(counts, 0)
    val = torch.rand(key.numel(), dtype=torch.float64, device="cuda", generator=gen) * 2.0 - 1.0
    return DeviceCSR(n, cols, key.numel(), rowptr.to(torch.int32), c.to(torch.int32).contiguous(), val, 32)


def generate(kind: str, n: int, deg: int, seed: int, param: int = 0) -> DeviceCSR:
    """Seeded square n x n matrix of a family, generated on the device:
    banded (bandwidth `param`), rmat (n rounded to a power of two, quadrant
    probabilities 0.57/0.19/0.19/0.05), uniform, block (dense-block width
    `param`; min(deg, width) entries per row inside the row's block)."""
    import torch
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    dev = "cuda"
    if kind == "rmat":
        scale = max(1, int(round(math.log2(n))))
        n = 1 << scale
        m = n * deg
        r = torch.zeros(m, dtype=torch.int64, device=dev)
        c = torch.zeros(m, dtype=torch.int64, device=dev)
        a, b, cc = 0.57, 0.19, 0.19
        for _ in range(scale):
            u = torch.rand(m, device=dev, generator=gen)
            down = u >= a + b
            right = ((u >= a) & (u < a + b)) | (u >= a + b + cc)
            r = r * 2 + down.to(torch.int64)
            c = c * 2 + right.to(torch.int64)
        return _csr(n, n, r, c, gen)
    rows = torch.arange(n, device=dev, dtype=torch.int64)
    if kind == "banded":
        bw = max(1, param)
        r = rows.repeat_interleave(deg)
        c = r + torch.randint(-bw, bw + 1, (r.numel(),), device=dev, generator=gen)
        keep = (c >= 0) & (c < n)
        return _csr(n, n, r[keep], c[keep], gen)
    if kind == "uniform":
        r = rows.repeat_interleave(deg)
        c = torch.randint(0, n, (r.numel(),), device=dev, generator=gen)
        return _csr(n, n, r, c, gen)
    if kind == "block":
        w = max(1, param)
        d = min(deg, w)
        r = rows.repeat_interleave(d)
        base = (r // w) * w
        c = base + torch.randint(0, w, (r.numel(),), device=dev, generator=gen)
        keep = c < n
        return _csr(n, n, r[keep], c[keep], gen)
    raise ValueError(kind)


@dataclass
class Spec:
    kind: str
    n: int
    deg: int
    param: int
    seed: int


def training_specs(count: int, seed: int, n_lo: int = 16384, n_hi: int = 1 << 20, deg_lo: int = 4,
                   deg_hi: int = 32) -> List[Spec]:
    """`count` seeded problems: families in turn, n log-uniform in [n_lo, n_hi],
    deg uniform in [deg_lo, deg_hi], bandwidth 3..65, block width 32..256."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = FAMILIES[i % len(FAMILIES)]
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        deg = int(rng.integers(deg_lo, deg_hi + 1))
        param = int(rng.integers(3, 66)) if kind == "banded" else int(rng.integers(32, 257)) if kind == "block" else 0
        out.append(Spec(kind, n, deg, param, int(rng.integers(1, 2 ** 31 - 1))))
    return out


def dataset(g: SpGEMM, specs: List[Spec], rows_per_matrix: int = 4096, min_products: int = 128, seed: int = 0):
    """(features, targets) of rows with more than min_products products, at
    most rows_per_matrix per problem, targets log2(1 + exact count)."""
    import torch
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    fs, ts = [], []
    thresh = math.log2(1.0 + min_products) + 1e-4
    for sp in specs:
        A = generate(sp.kind, sp.n, sp.deg, sp.seed, sp.param)
        feat = features(g, A)
        cnt = g.symbolic(A, A).view(torch.int32).to(torch.int64) & 0xFFFFFFFF
        sel = torch.nonzero(feat[:, 1] > thresh).flatten()
        if sel.numel() > rows_per_matrix:
            sel = sel[torch.randperm(sel.numel(), device="cuda", generator=gen)[:rows_per_matrix]]
        if sel.numel():
            fs.append(feat.index_select(0, sel))
            ts.append(torch.log2(1.0 + cnt.index_select(0, sel).double()).float())
        del A, feat, cnt
    if not fs:
        return (torch.empty((0, MLP_FEATURES), dtype=torch.float32, device="cuda"),
                torch.empty(0, dtype=torch.float32, device="cuda"))
    return torch.cat(fs).contiguous(), torch.cat(ts).contiguous()
