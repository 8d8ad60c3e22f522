"""CPU tests of the estimator oracle: BF16 rounding, and the float64 analytic
gradient against central finite differences (which pins the backward
formulas the library's kernels are checked against)."""
import numpy as np

from oracle import mlp as N


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0], np.float32)
    r = N.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0) wins;
    # 1 + 3*2^-8 is a tie between 1 + 2^-7 and 1 + 2^-6: 1 + 2^-6 (even) wins
    assert list(r) == [1.0, 1.0, 1.0 + 2 ** -6, 1.0, -2.5, 0.0]


def test_float64_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    params = N.init_params(seed=4).astype(np.float64)
    params[N.OFF_B1:N.OFF_W2] = rng.normal(0, 0.1, N.H)
    params[N.OFF_B2:N.OFF_W3] = rng.normal(0, 0.1, N.H)
    mu = rng.normal(0, 1, N.F)
    isd = rng.uniform(0.5, 2.0, N.F)
    feat = rng.normal(0, 1, (40, N.F))
    target = rng.normal(0, 1, 40)
    g, _ = N.grad(params, mu, isd, feat, target, 40.0, rounding=False)
    idx = np.concatenate([rng.choice(np.arange(N.OFF_W1, N.OFF_B1), 12, replace=False),
                          rng.choice(np.arange(N.OFF_W2, N.OFF_B2), 12, replace=False),
                          np.arange(N.OFF_B1, N.OFF_B1 + 4), np.arange(N.OFF_B2, N.OFF_B2 + 4),
                          np.arange(N.OFF_W3, N.OFF_W3 + 6), [N.OFF_B3]])
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (N.loss(p1, mu, isd, feat, target, 40.0) - N.loss(p2, mu, isd, feat, target, 40.0)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_rounded_gradient_close_to_float64():
    rng = np.random.default_rng(5)
    params = N.init_params(seed=6)
    mu = np.zeros(N.F, np.float32)
    isd = np.ones(N.F, np.float32)
    feat = rng.normal(0, 1, (256, N.F)).astype(np.float32)
    target = rng.normal(0, 1, 256).astype(np.float32)
    g32, _ = N.grad(params, mu, isd, feat, target, 256.0, rounding=True)
    g64, _ = N.grad(params.astype(np.float64), mu, isd, feat, target, 256.0, rounding=False)
    assert np.linalg.norm(g32 - g64) <= 0.05 * np.linalg.norm(g64)
