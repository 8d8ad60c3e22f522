"""GPU parity tests: the sm_100a library (through the C ABI) against the CPU
oracle on the same seeded inputs. Structure must match bit for bit; values
within |x - y| <= 1e-12 * sum_k |a_ik * b_kj| (FP64; summation order differs)."""
import numpy as np
import pytest

from oracle import oracle as O
from research_b200 import matrices as M
from research_b200.ocean import DeviceCSR, HostCSR, OceanError, SpGEMM

pytestmark = pytest.mark.gpu

TOL = 1e-12
SYM_BINS = {"esc1": 0, "esc2": 1, "esc4": 2, "hash_s": 3, "hash_m": 4, "hash_l": 5, "bitmap": 6}
NUM_BINS = {"esc1": 0, "esc2": 1, "esc4": 2, "hash_s": 3, "hash_m": 4, "hash_l": 5, "bitmap": 6}


def multiply_device(A, B, config=None):
    g = SpGEMM(config or {})
    dA = DeviceCSR.from_host(A)
    dB = dA if B is A else DeviceCSR.from_host(B)
    C = g.multiply(dA, dB)
    h = C.download()
    C.free()
    return h, g.get_stats()


def check(A, B, C, tol=TOL):
    cp, cj, cx, ca = O.spgemm(A, B, with_abs=True)
    assert C.rows == A.rows and C.cols == B.cols
    assert int(C.rowptr[-1]) == C.nnz == int(cp[-1])
    return O.compare(C.rowptr, C.col, C.val, cp, cj, cx, ca, tol)


def test_tiny_cases_device_and_host(tiny_cases):
    for name, A, B, (rp, col, val) in tiny_cases:
        C, _ = multiply_device(A, B)
        O.compare(C.rowptr, C.col, C.val, rp, col, val, tol=0.0)
        H = SpGEMM().multiply(A, B)
        O.compare(H.rowptr, H.col, H.val, rp, col, val, tol=0.0)


@pytest.mark.parametrize("sym", list(SYM_BINS))
@pytest.mark.parametrize("num", list(NUM_BINS))
def test_tiny_cases_every_class(tiny_cases, sym, num):
    cfg = {"force_sym_bin": SYM_BINS[sym], "force_num_bin": NUM_BINS[num]}
    for name, A, B, (rp, col, val) in tiny_cases:
        C, _ = multiply_device(A, B, cfg)
        O.compare(C.rowptr, C.col, C.val, rp, col, val, tol=0.0)


def test_laplacian_256_full():
    A = M.laplacian_2d(256, 256, seed=0)
    C, st = multiply_device(A, A)
    check(A, A, C)
    assert st["C"]["nnz"] == 846852 and st["stats"]["intermediate_product"] == 1629192


@pytest.mark.parametrize("sym", ["esc4", "hash_s", "hash_m", "hash_l", "bitmap"])
@pytest.mark.parametrize("num", ["esc4", "hash_s", "hash_m", "hash_l", "bitmap"])
def test_forced_classes_uniform(sym, num):
    A = M.uniform_random(6000, 10, seed=11)
    # keep every row within the forced classes' capacities
    prod, _, _ = O.row_stats(A, A)
    cnt = O.symbolic(A, A)
    caps_sym = {"esc4": 128, "hash_s": 1024, "hash_m": 4096, "hash_l": 16384, "bitmap": 1 << 40}
    caps_num = {"esc4": 128, "hash_s": 512, "hash_m": 2048, "hash_l": 4096, "bitmap": 1 << 40}
    if prod.max() > caps_sym[sym] or cnt.max() > caps_num[num] or (num == "esc4" and prod.max() > 128):
        pytest.skip("matrix exceeds the forced class capacity")
    C, _ = multiply_device(A, A, {"force_sym_bin": SYM_BINS[sym], "force_num_bin": NUM_BINS[num]})
    check(A, A, C)


@pytest.mark.parametrize("readback", [False, True])
@pytest.mark.parametrize("gen", ["uniform", "banded", "block", "rmat14", "rect"])
def test_families(gen, readback):
    if gen == "uniform":
        A = M.uniform_random(20000, 16, seed=1); B = A
    elif gen == "banded":
        A = M.banded(30000, 65, 24, seed=2); B = A
    elif gen == "block":
        A = M.block_diagonal(32768, 256, 32, seed=3); B = A
    elif gen == "rmat14":
        A = M.rmat(14, 16, seed=4); B = A
    else:
        A = M.rect_poisson(16384, 65536, 12.0, seed=5); B = M.transpose(A)
    # readback: class sizes read back after the analysis (selective launches, bitmap cache);
    # otherwise the small-input mode that launches every class without a read-back
    C, st = multiply_device(A, B, {"small_problem_nnz": 0 if readback else 1 << 30})
    check(A, B, C)
    assert sum(st["binning_2"]) == int(np.count_nonzero(np.diff(C.rowptr.astype(np.int64))))


def test_rect_aat_full_size():
    A = M.rect_poisson(262144, 1048576, 12.0, seed=0)
    At = M.transpose(A)
    C, st = multiply_device(A, At)
    check(A, At, C)


def test_rmat_scale16_full():
    A = M.rmat(16, 16, seed=0)
    C, st = multiply_device(A, A)
    check(A, A, C)


def test_wide_span_multi_window():
    # rows whose output span exceeds one 2^20-column bitmap window
    n = 3 * (1 << 20) + 17
    rng = np.random.default_rng(5)
    rows = 64
    r = np.repeat(np.arange(rows), 40)
    c = rng.integers(0, n, r.size)
    B = M.from_coo(rows, n, r, c, rng.uniform(-1, 1, r.size))
    A = M.from_coo(200, rows, np.repeat(np.arange(200), 24), rng.integers(0, rows, 200 * 24),
                   rng.uniform(-1, 1, 200 * 24))
    for num in ("bitmap", None):
        cfg = {"force_sym_bin": SYM_BINS["bitmap"]} if num else {}
        if num:
            cfg["force_num_bin"] = NUM_BINS["bitmap"]
        C, _ = multiply_device(A, B, cfg)
        check(A, B, C)


def test_hub_rows_large_products():
    # a few rows with very many products and outputs (bitmap class)
    rng = np.random.default_rng(8)
    n = 1 << 17
    B = M.uniform_random(n, 40, seed=8)
    r = np.concatenate([np.repeat(np.arange(4), 3000), np.repeat(np.arange(4, 300), 5)])
    A = M.from_coo(300, n, r, rng.integers(0, n, r.size), rng.uniform(-1, 1, r.size))
    C, st = multiply_device(A, B)
    check(A, B, C)
    assert st["binning_2"][NUM_BINS["bitmap"]] >= 4


def test_rowptr_64_and_mixed_inputs():
    A = M.rmat(12, 8, seed=6)
    A64 = A.widened()
    for a, b in ((A64, A64), (A64, A), (A, A64)):
        C, _ = multiply_device(a, b)
        check(A, A, C)
    C, st = multiply_device(A, A, {"output_rowptr_bits": 64})
    assert C.rowptr.dtype == np.uint64 and st["decision"]["rowptr_bits"] == 64
    check(A, A, C)


def test_empty_inputs():
    z = HostCSR(0, 5, np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros(0))
    B = M.uniform_random(5, 2, seed=1)
    C, _ = multiply_device(z, B)
    assert C.rows == 0 and C.nnz == 0 and C.rowptr.tolist() == [0]
    E = HostCSR(7, 5, np.zeros(8, np.uint32), np.zeros(0, np.uint32), np.zeros(0))
    C, _ = multiply_device(E, B)
    assert C.nnz == 0 and C.rowptr.tolist() == [0] * 8
    Bz = HostCSR(5, 9, np.zeros(6, np.uint32), np.zeros(0, np.uint32), np.zeros(0))
    A = M.from_coo(4, 5, [0, 1, 3], [1, 2, 4], [1.0, 2.0, 3.0])
    C, _ = multiply_device(A, Bz)
    assert C.nnz == 0


def test_last_row_end_taken_from_nnz():
    # rowptr[rows] is not read (reference: src/CSR.cpp:54); poison it
    A = M.uniform_random(3000, 7, seed=12)
    bad = HostCSR(A.rows, A.cols, A.rowptr.copy(), A.col, A.val)
    bad.rowptr[-1] = 0xFFFFFFF0
    C, _ = multiply_device(bad, A)
    check(A, A, C)


def test_errors_are_status_codes():
    A = M.uniform_random(100, 3, seed=1)
    B = M.rect_poisson(50, 60, 3.0, seed=1)
    with pytest.raises(OceanError) as e:
        multiply_device(A, B)
    assert e.value.code == 4 and "Incompatible" in str(e.value)
    with pytest.raises(OceanError) as e:
        SpGEMM({"use_hybrid_accumulator": True, "use_indirect_sort": False}).multiply(A, A)
    assert e.value.code == 4
    # a row forced into a class too small for it is reported, not mis-written
    # (2048-column blocks: wider than the 1024 slots, so the rows are hashed)
    R = M.block_diagonal(8192, 2048, 64, seed=2)
    with pytest.raises(OceanError) as e:
        multiply_device(R, R, {"force_num_bin": NUM_BINS["hash_s"]})
    assert e.value.code in (2, 6)


def test_repeated_calls_reuse_handle():
    A = M.rmat(13, 8, seed=21)
    g = SpGEMM({"track_stage_time": True})
    dA = DeviceCSR.from_host(A)
    first = None
    for _ in range(3):
        C = g.multiply(dA, dA)
        h = C.download()
        C.free()
        if first is None:
            first = h
            check(A, A, h)
        else:
            assert np.array_equal(h.rowptr, first.rowptr) and np.array_equal(h.col, first.col)
    st = g.get_stats()
    assert st["total_time"] > 0 and st["timing"]["numeric"] >= 0 and st["gflops"] > 0
    assert g.stage_ms("symbolic") >= 0


def test_symbolic_entry_point():
    A = M.rmat(12, 8, seed=13)
    g = SpGEMM()
    dA = DeviceCSR.from_host(A)
    cnt = g.symbolic(dA, dA).cpu().numpy().view(np.uint32)
    assert np.array_equal(cnt.astype(np.uint64), O.symbolic(A, A))


def test_murmur3_device_matches_reference_kat(murmur_kat):
    import torch
    from research_b200.ocean import murmur3_device
    keys, hashes = murmur_kat
    out = murmur3_device(torch.from_numpy(keys.view(np.int32)).cuda(), 1234)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), hashes)


@pytest.mark.parametrize("frac", [0.0, 0.25])
def test_bitmap_cache_on_and_off(frac):
    # rows of the bitmap class either reload the bitmap saved by the symbolic
    # pass or mark their columns again; both must give the oracle's C
    A = M.rmat(15, 16, seed=3)
    C, st = multiply_device(A, A, {"bitmap_cache_fraction": frac, "small_problem_nnz": 0})
    check(A, A, C)
    used = st["decision"]["bitmap_cache_used_bytes"]
    assert (used > 0) == (frac > 0)


@pytest.mark.parametrize("k", [1, 2, 4])
def test_esc_classes_with_repeated_columns(k):
    # rows whose products repeat the same column many times, across register
    # rows of the warp sort (runs longer than 32), and cancelling sums
    rng = np.random.default_rng(40 + k)
    n = 64
    cap = 32 * k
    B = M.from_coo(n, 50, np.repeat(np.arange(n), 3), rng.integers(0, 6, 3 * n), rng.uniform(-1, 1, 3 * n))
    nb = np.diff(B.rowptr.astype(np.int64))
    rows, cols = [], []
    for i in range(300):
        budget = int(rng.integers(1, cap + 1))
        picked, tot = [], 0
        for j in rng.permutation(n):
            if tot + nb[j] > budget:
                continue
            picked.append(j)
            tot += nb[j]
        rows += [i] * len(picked)
        cols += picked
    A = M.from_coo(300, n, rows, cols, rng.uniform(-1, 1, len(rows)))
    cls = {1: "esc1", 2: "esc2", 4: "esc4"}[k]
    C, st = multiply_device(A, B, {"force_sym_bin": SYM_BINS[cls], "force_num_bin": NUM_BINS[cls]})
    check(A, B, C)


def test_esc_overflow_is_reported():
    A = M.block_diagonal(2048, 256, 32, seed=5)  # 1024 products per row
    with pytest.raises(OceanError) as e:
        multiply_device(A, A, {"force_sym_bin": SYM_BINS["esc4"]})
    assert e.value.code in (2, 6)
