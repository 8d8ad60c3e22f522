"""CPU oracle of the learned row-size estimator — TEST INFRASTRUCTURE ONLY.

Only tests/ may import this module, as the checker of libocean.so's
estimator kernels (ocean_mlp_forward / ocean_mlp_grad). The product path never
calls it. The reference has no learned estimator, so there is no reference file
to follow; this restates the network the library defines:

    x  = bf16((f - mu) * inv_sd)                      f: 16 raw features
    z1 = x  W1^T + b1,   h1 = bf16(relu(z1))          W1 [64][16]
    z2 = h1 W2^T + b2,   h2 = bf16(relu(z2))          W2 [64][64]
    y  = h2 . w3 + b3                                 w3 [64]
    L  = sum_i (y_i - t_i)^2 / batch

with weights rounded to BF16 where the tensor cores use them and FP32
everywhere else. The backward pass rounds dZ2 and dZ1 to BF16 where they feed
the tensor cores, as the library does. ``rounding=False`` gives the same
network in float64 without any rounding; its gradient is pinned against
central finite differences in tests/test_oracle_mlp.py.
"""
from __future__ import annotations

import numpy as np

F, H = 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
P = OFF_B3 + 1
BLOB = P + 2 * F + 1


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even); float32 result."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(x.shape)


def unpack(params):
    p = np.asarray(params)
    return (p[OFF_W1:OFF_B1].reshape(H, F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initial weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(P, np.float32)
    p[OFF_W1:OFF_B1] = rng.normal(0, np.sqrt(2.0 / F), H * F)
    p[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2.0 / H), H * H)
    p[OFF_W3:OFF_B3] = rng.normal(0, np.sqrt(1.0 / H), H)
    return p


def _mm(a, b, rounding):
    # products summed in float64, then stored in the working precision
    r = np.asarray(a, np.float64) @ np.asarray(b, np.float64)
    return r.astype(np.float32) if rounding else r


def forward(params, mu, inv_sd, feat, rounding: bool = True):
    """Returns (y, cache) for feat[n][16]."""
    dt = np.float32 if rounding else np.float64
    rb = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    W1, b1, W2, b2, w3, b3 = [np.asarray(v, dt) for v in unpack(params)]
    f = np.asarray(feat, dt)
    x = rb((f - np.asarray(mu, dt)) * np.asarray(inv_sd, dt))
    z1 = _mm(x, rb(W1).T, rounding) + b1
    h1 = rb(np.maximum(z1, 0))
    z2 = _mm(h1, rb(W2).T, rounding) + b2
    h2 = rb(np.maximum(z2, 0))
    y = _mm(h2, rb(w3)[:, None], rounding)[:, 0] + b3
    return y, (x, z1, h1, z2, h2, W2, w3)


def grad(params, mu, inv_sd, feat, target, batch, rounding: bool = True):
    """(gradient of sum (y - t)^2 / batch over the params, sum of squared errors)."""
    dt = np.float32 if rounding else np.float64
    rb = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    y, (x, z1, h1, z2, h2, W2, w3) = forward(params, mu, inv_sd, feat, rounding)
    diff = y - np.asarray(target, dt)
    dy = (dt(2.0) * diff) * dt(1.0 / batch) if rounding else 2.0 * diff / batch
    g = np.zeros(P, np.float64)
    g[OFF_B3] = dy.sum(dtype=np.float64)
    g[OFF_W3:OFF_B3] = (np.asarray(dy, np.float64)[:, None] * h2).sum(0)
    dz2 = dy[:, None] * rb(w3)[None, :] * (z2 > 0)
    g[OFF_B2:OFF_W3] = dz2.sum(0, dtype=np.float64)
    dz2r = rb(dz2)
    dh1 = _mm(dz2r, rb(W2), rounding)
    dz1 = dh1 * (z1 > 0)
    g[OFF_B1:OFF_W2] = dz1.sum(0, dtype=np.float64)
    dz1r = rb(dz1)
    g[OFF_W2:OFF_B2] = (np.asarray(dz2r, np.float64).T @ np.asarray(h1, np.float64)).reshape(-1)
    g[OFF_W1:OFF_B1] = (np.asarray(dz1r, np.float64).T @ np.asarray(x, np.float64)).reshape(-1)
    return g, float((np.asarray(diff, np.float64) ** 2).sum())


def loss(params, mu, inv_sd, feat, target, batch, rounding: bool = False) -> float:
    y, _ = forward(params, mu, inv_sd, feat, rounding)
    return float(((np.asarray(y, np.float64) - np.asarray(target, np.float64)) ** 2).sum() / batch)
