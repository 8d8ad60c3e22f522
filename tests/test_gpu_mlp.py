"""Learned row-size estimator on the GPU: the tensor-core forward and backward
kernels against the CPU oracle (oracle/mlp.py), the feature kernel against the
CPU restatements, a training run that must fit, and the learned estimation
workflow, which must give exactly the oracle's C whatever the estimates."""
import math

import numpy as np
import pytest

from oracle import mlp as N
from oracle import oracle as O
from oracle import segmentation as S
from research_b200 import estimator as E
from research_b200 import matrices as M
from research_b200.ocean import DeviceCSR, SpGEMM

pytestmark = pytest.mark.gpu


def random_net(seed):
    rng = np.random.default_rng(seed)
    p = N.init_params(seed)
    p[N.OFF_B1:N.OFF_W2] = rng.normal(0, 0.2, N.H)
    p[N.OFF_B2:N.OFF_W3] = rng.normal(0, 0.2, N.H)
    p[N.OFF_B3] = 0.3
    mu = rng.normal(0, 1, N.F).astype(np.float32)
    isd = rng.uniform(0.5, 1.5, N.F).astype(np.float32)
    return p, mu, isd


def feats(n, seed):
    return np.random.default_rng(seed).normal(0, 1.5, (n, N.F)).astype(np.float32)


@pytest.mark.parametrize("n", [37, 1000, 80000])
def test_forward_matches_oracle(n):
    import torch
    p, mu, isd = random_net(1)
    f = feats(n, 2)
    net = E.Network(p, mu, isd)
    g = SpGEMM()
    got = net.forward(g, torch.from_numpy(f).cuda()).cpu().numpy()
    want, _ = N.forward(p, mu, isd, f)
    err = np.abs(got - want)
    # BF16 activations: an accumulation-order difference can flip one rounding
    assert np.median(err) < 1e-4
    assert err.max() < 2e-2 * (1 + np.abs(want).max())


@pytest.mark.parametrize("n", [1000, 80000])
def test_gradient_matches_oracle(n):
    import torch
    p, mu, isd = random_net(3)
    f = feats(n, 4)
    t = np.random.default_rng(5).normal(0, 1, n).astype(np.float32)
    net = E.Network(p, mu, isd)
    g = SpGEMM()
    gbuf = torch.zeros(N.P, dtype=torch.float32, device="cuda")
    lbuf = torch.zeros(1, dtype=torch.float32, device="cuda")
    net.grad(g, torch.from_numpy(f).cuda(), torch.from_numpy(t).cuda(), float(n), gbuf, lbuf)
    got = gbuf.cpu().numpy().astype(np.float64)
    want, loss = N.grad(p, mu, isd, f, t, float(n))
    blocks = {"W1": (N.OFF_W1, N.OFF_B1), "b1": (N.OFF_B1, N.OFF_W2), "W2": (N.OFF_W2, N.OFF_B2),
              "b2": (N.OFF_B2, N.OFF_W3), "w3": (N.OFF_W3, N.OFF_B3), "b3": (N.OFF_B3, N.P)}
    # the oracle rounds the activations and operands to BF16 where the kernels
    # do, so only accumulation order (and a rare flipped BF16 rounding) differs
    rels = {}
    for name, (a, b) in blocks.items():
        rels[name] = float(np.linalg.norm(got[a:b] - want[a:b]) / max(np.linalg.norm(want[a:b]), 1e-12))
    print("gradient relative error per block:", rels)
    assert all(r < 5e-3 for r in rels.values()), rels
    assert abs(float(lbuf.item()) - loss) <= 1e-3 * loss


def test_training_fits_a_smooth_target():
    import torch
    rng = np.random.default_rng(7)
    n = 60000
    f = rng.normal(0, 1, (n, N.F)).astype(np.float32)
    t = (0.8 * f[:, 0] - 0.5 * np.abs(f[:, 1]) + np.maximum(f[:, 2] + f[:, 3], 0) + 2.0).astype(np.float32)
    mu = np.zeros(N.F, np.float32)
    isd = np.ones(N.F, np.float32)
    net = E.Network.initial(mu, isd, seed=8)
    g = SpGEMM()
    ft, tt = torch.from_numpy(f).cuda(), torch.from_numpy(t).cuda()
    before = float(((net.forward(g, ft) - tt) ** 2).mean().item())
    E.train(g, net, ft, tt, steps=600, batch=4096, lr=3e-3, seed=9, log_every=100)
    after = float(((net.forward(g, ft) - tt) ** 2).mean().item())
    assert after < 0.05 * before and after < 0.05, (before, after)


def test_features_match_restatements():
    import torch
    A = M.rmat(11, 8, seed=10)
    g = SpGEMM()
    dA = DeviceCSR.from_host(A)
    got = E.features(g, dA).cpu().numpy()
    prod, lo, hi, anz, maxb = S.row_stats(A, A)
    sk = O.hll_sketch_rows(A, 5)
    hll = np.array([O.hll_estimate_union(sk, 5, A.col[A.rowptr[r]:A.rowptr[r + 1]].astype(np.uint32))
                    for r in range(A.rows)], np.float64)
    span = np.where(prod > 0, hi - lo + 1, 0)
    ub = np.minimum(prod, span)
    lg = lambda x: np.log2(1.0 + np.asarray(x, np.float64))
    want = np.zeros((A.rows, 16))
    want[:, 0], want[:, 1], want[:, 2], want[:, 3] = lg(anz), lg(prod), lg(span), lg(maxb)
    want[:, 4], want[:, 5] = lg(ub), lg(hll)
    want[:, 6], want[:, 7] = want[:, 1] - want[:, 0], want[:, 5] - want[:, 4]
    want[:, 8], want[:, 9] = math.log2(1 + A.cols), math.log2(1 + A.nnz / A.rows)
    want[:, 10] = want[:, 3] - want[:, 4]
    assert np.allclose(got, want, atol=2e-5, rtol=1e-5)


def quick_network(tmp_path):
    """A network trained for a few seconds on small products of every family."""
    g = SpGEMM()
    specs = E.training_specs(24, seed=11, n_lo=8192, n_hi=65536)
    f, t = E.dataset(g, specs, rows_per_matrix=2048, seed=12)
    mu, isd = E.normalisation(f)
    net = E.Network.initial(mu, isd, seed=13)
    E.train(g, net, f, t, steps=400, batch=4096, lr=3e-3, seed=14)
    E.calibrate_margin(g, net, f, t, 0.95)
    path = tmp_path / "net.txt"
    net.save(path)
    return path, net


@pytest.mark.parametrize("margin_scale", [1.0, 0.0])
def test_learned_workflow_is_exact(tmp_path, margin_scale):
    path, _ = quick_network(tmp_path)
    for A in (M.rmat(14, 12, seed=15), M.banded(30000, 40, 24, seed=16), M.block_diagonal(20000, 128, 24, seed=17)):
        g = SpGEMM({"use_learned_estimator": True, "learned_estimator_weights": str(path), "force_workflow": 1,
                    "learned_margin_scale": margin_scale, "estimator_metrics": True})
        C = g.multiply(A, A)
        rp, cj, cx, ca = O.spgemm(A, A, with_abs=True)
        O.compare(C.rowptr, C.col, C.val, rp, cj, cx, ref_abs=ca)
        est = g.get_stats()["estimation"]
        assert est["estimator"] == "learned"
        assert est["metrics"]["rows"] > 0
        if margin_scale == 0.0:
            assert est["overflow_rows"] > 0  # no margin: some rows must have been rerun


def test_weights_file_round_trip(tmp_path):
    p, mu, isd = random_net(20)
    net = E.Network(p, mu, isd, margin=0.375)
    net.save(tmp_path / "w.txt")
    back = E.Network.load(tmp_path / "w.txt")
    assert np.array_equal(back.blob(), net.blob())
