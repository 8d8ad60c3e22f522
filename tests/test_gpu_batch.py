"""Batched products on the GPU: every result of a batch plan (one captured
graph per run) and of the one-shot batched call equals the oracle's product
of that problem alone, over mixed families and sizes, square and rectangular,
32- and 64-bit row pointers, empty problems, every workflow, the learned
estimator, the autotuner, changed values between runs, and a changed
structure (detected, nothing written out of bounds)."""
import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import Batch, DeviceCSR, HostCSR, OceanError, SpGEMM, spgemm_batched

pytestmark = pytest.mark.gpu


def mixed_problems(count, seed, n_lo=500, n_hi=6000):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        d = int(rng.integers(4, 33))
        k = i % 4
        if k == 0:
            out.append(M.banded(n, int(rng.integers(3, 66)), d, seed=seed + i))
        elif k == 1:
            out.append(M.rmat(max(9, int(np.log2(n))), d, seed=seed + i))
        elif k == 2:
            out.append(M.uniform_random(n, d, seed=seed + i))
        else:
            out.append(M.block_diagonal(n, int(rng.integers(32, 257)), d, seed=seed + i))
    return out


def check(results, As, Bs=None):
    assert len(results) == len(As)
    for p, (C, A) in enumerate(zip(results, As)):
        B = A if Bs is None else Bs[p]
        h = C.download()
        rp, cj, cx, ca = O.spgemm(A, B, with_abs=True)
        assert h.rows == A.rows and h.cols == B.cols
        O.compare(h.rowptr, h.col, h.val, rp, cj, cx, ref_abs=ca)


@pytest.mark.parametrize("cfg", [{}, {"force_workflow": 0}, {"force_workflow": 1}, {"force_workflow": 2},
                                 {"use_learned_estimator": True}])
def test_batch_plan_matches_each_product(cfg):
    As = mixed_problems(24, seed=100)
    dA = [DeviceCSR.from_host(a) for a in As]
    g = SpGEMM(cfg)
    b = Batch(g, dA)
    info = b.info()
    assert info["problems"] == 24 and info["graph"] is True
    check(b.run(), As)
    check(b.run(), As)  # a second launch of the same graph


def test_batch_rectangular_general_b_and_64bit():
    rng = np.random.default_rng(5)
    As, Bs = [], []
    for i in range(9):
        r, c = int(rng.integers(200, 3000)), int(rng.integers(200, 3000))
        A = M.rect_poisson(r, c, float(rng.uniform(2, 12)), seed=200 + i)
        B = M.transpose(M.rect_poisson(int(rng.integers(100, 2000)), c, 6.0, seed=300 + i))
        if i % 3 == 0:
            A = A.widened()
        As.append(A)
        Bs.append(B)
    g = SpGEMM()
    dA = [DeviceCSR.from_host(a) for a in As]
    dB = [DeviceCSR.from_host(x) for x in Bs]
    check(Batch(g, dA, dB).run(), As, Bs)
    check(spgemm_batched(g, dA, dB), As, Bs)


def test_batch_with_empty_problems():
    empty = HostCSR(0, 0, np.zeros(1, np.uint32), np.empty(0, np.uint32), np.empty(0))
    no_entries = HostCSR(50, 50, np.zeros(51, np.uint32), np.empty(0, np.uint32), np.empty(0))
    As = [empty, M.uniform_random(300, 5, seed=1), no_entries, M.laplacian_2d(20, 20), empty]
    g = SpGEMM()
    dA = [DeviceCSR.from_host(a) for a in As]
    res = Batch(g, dA).run()
    check(res, As)
    assert res[0].nnz == 0 and res[2].nnz == 0
    only_empty = [DeviceCSR.from_host(empty), DeviceCSR.from_host(no_entries)]
    res = Batch(g, only_empty).run()
    assert [r.nnz for r in res] == [0, 0]
    assert list(res[1].download().rowptr) == [0] * 51


def test_autotuned_learned_batch():
    As = mixed_problems(16, seed=400, n_hi=20000)
    dA = [DeviceCSR.from_host(a) for a in As]
    g = SpGEMM({"use_learned_estimator": True, "batch_autotune": True})
    b = Batch(g, dA)
    info = b.info()
    assert info["estimator"] == "learned" and info["tuned_ms"] > 0 and "esc_max_products" in info["tuning"]
    check(b.run(), As)


def test_values_change_between_runs():
    import torch
    As = mixed_problems(8, seed=500)
    dA = [DeviceCSR.from_host(a) for a in As]
    g = SpGEMM({"use_learned_estimator": True})
    b = Batch(g, dA)
    check(b.run(), As)
    for a, d in zip(As, dA):
        a.val[:] = a.val * 2.0 - 0.5
        d.val.copy_(torch.from_numpy(a.val).cuda())
    check(b.run(), As)


def test_structure_change_is_detected():
    import torch
    As = [M.uniform_random(2000, 8, seed=600), M.banded(3000, 10, 8, seed=601)]
    dA = [DeviceCSR.from_host(a) for a in As]
    g = SpGEMM({"force_workflow": 0})
    b = Batch(g, dA)
    check(b.run(), As)
    # scatter the banded problem's columns over the whole range: more output
    # per row than planned; the run must refuse and write nothing out of bounds
    rng = np.random.default_rng(7)
    rp = As[1].rowptr.astype(np.int64)
    cols = np.empty(As[1].nnz, np.uint32)
    for r in range(As[1].rows):
        k = int(rp[r + 1] - rp[r])
        cols[rp[r]:rp[r + 1]] = np.sort(rng.choice(3000, size=k, replace=False))
    new_col = torch.from_numpy(cols.view(np.int32)).cuda()
    dA[1].col.copy_(new_col)
    with pytest.raises(OceanError) as e:
        b.run()
    assert e.value.code == 4 and "structure changed" in str(e.value)
    # the handle and the device stay usable
    check([g.multiply(dA[0], dA[0])], As[:1])


def test_one_shot_results_are_owned():
    As = mixed_problems(6, seed=700)
    g = SpGEMM()
    res = spgemm_batched(g, [DeviceCSR.from_host(a) for a in As])
    check(res, As)
    for r in res:
        r.free()


def test_autotune_cache_round_trip(tmp_path):
    # the first plan searches and appends its knobs to the cache file; a
    # second plan of the same batch takes them from the cache without searching
    cache = tmp_path / "tune.jsonl"
    As = mixed_problems(12, seed=300)
    dA = [DeviceCSR.from_host(a) for a in As]
    cfg = {"batch_autotune": True, "autotune_cache_file": str(cache)}
    g1 = SpGEMM(cfg)
    p1 = Batch(g1, dA)
    i1 = p1.info()
    assert i1["tune_cached"] is False and cache.exists()
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and i1["tune_key"] in lines[0]
    g2 = SpGEMM(cfg)
    p2 = Batch(g2, dA)
    i2 = p2.info()
    assert i2["tune_cached"] is True and i2["tune_key"] == i1["tune_key"]
    for k in ("esc_max_products", "hash_s_max_scale", "bitmap_words_scale", "prefer_direct_hash", "numeric_windows"):
        assert i2[k] == i1[k]
    assert len(cache.read_text().splitlines()) == 1
    check(p2.run(), As)
    # a damaged line is skipped, and another batch gets its own key
    with open(cache, "a") as f:
        f.write("{not json\n")
    Bs = mixed_problems(5, seed=301)
    p3 = Batch(SpGEMM(cfg), [DeviceCSR.from_host(a) for a in Bs])
    assert p3.info()["tune_cached"] is False
    check(p3.run(), Bs)
    for p in (p1, p2, p3):
        p.close()
