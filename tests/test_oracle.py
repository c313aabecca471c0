"""CPU checks of the oracle (the checker itself): generators against glibc,
restatements against each other and against the exact-math oracle, and the
committed golden fixtures."""
import ctypes
import json
import glob
import os

import numpy as np
import pytest

from oracle import oracle as orc
from tests._util import componentwise_err, fp32_bound, normwise_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _glibc():
    libc = ctypes.CDLL("libc.so.6")
    libc.srand48.argtypes = [ctypes.c_long]
    libc.drand48.restype = ctypes.c_double
    return libc


@pytest.mark.parametrize("seed", [0, 1, 17, 123456789])
def test_drand48_matches_glibc(seed):
    libc = _glibc()
    libc.srand48(seed)
    want = np.array([libc.drand48() for _ in range(1000)])
    got = orc.drand48(seed, 1000)
    assert np.array_equal(got, want)
    # jump-ahead agrees with sequential draws
    assert np.array_equal(orc.drand48(seed, 10, skip=990), want[990:])


def test_uniform_matches_reference_random_matrix():
    # random_matrix(): a[i*n+j] = 2.0 * (float)drand48() - 1.0 stored to float
    # (benchmark/small_SGEMM/LibShalom_sgemm.c:26-34)
    libc = _glibc()
    libc.srand48(0)
    want = np.empty(500, np.float32)
    for i in range(500):
        f = np.float32(libc.drand48())
        want[i] = np.float32(2.0 * np.float64(f) - 1.0)
    got = orc.uniform_f32(0, 500)
    assert np.array_equal(got, want)
    assert got.min() >= -1.0 and got.max() < 1.0


@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (5, 16, 8), (7, 9, 13), (80, 80, 80),
                                   (33, 17, 65)])
def test_kseq_within_fp32_bound(M, N, K, transb):
    A, B = orc.gemm_inputs_f32(3, M, N, K, transb)
    ref = orc.sgemm_f64(A, B, transb)
    C = orc.sgemm_kseq(A, B, transb)
    ab = orc.sgemm_absprod(A, B, transb)
    assert componentwise_err(C, ref, ab) <= fp32_bound(K)


@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (5, 16, 8), (7, 9, 13), (80, 80, 80),
                                   (6, 37, 3), (130, 70, 33)])
def test_port_equals_kseq(M, N, K, transb):
    # the 5x16-tile CPU port keeps the k-sequential FMA order of the reference
    A, B = orc.gemm_inputs_f32(5, M, N, K, transb)
    assert np.array_equal(orc.port_sgemm(A, B, transb), orc.sgemm_kseq(A, B, transb))


@pytest.mark.parametrize("threads", [1, 4, 8])
@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("M,N,K", [(64, 300, 700), (300, 20, 641), (33, 65, 320)])
def test_port_mp_equals_kblocked(M, N, K, transb, threads):
    A, B = orc.gemm_inputs_f32(9, M, N, K, transb)
    got = orc.port_sgemm_mp(A, B, transb, threads)
    assert np.array_equal(got, orc.sgemm_kseq(A, B, transb, kblock=320))


def test_port_dgemm_equals_kseq():
    rng = np.random.default_rng(0)
    for (M, N, K) in [(5, 5, 5), (22, 13, 32), (7, 6, 4), (32, 32, 32), (1, 9, 26)]:
        A = rng.standard_normal((M, K))
        B = rng.standard_normal((K, N))
        assert np.array_equal(orc.port_dgemm(A, B), orc.dgemm_kseq(A, B, 0))


def test_nt_reforder_close_to_kseq():
    A, B = orc.gemm_inputs_f32(0, 80, 80, 80, 1)
    r = orc.sgemm_nt_reforder(A, B)
    k = orc.sgemm_kseq(A, B, 1)
    # rows >= 5 of every strip use the k-sequential KERNEL5x16 order
    assert np.array_equal(r[5:], k[5:])
    ref = orc.sgemm_f64(A, B, 1)
    ab = orc.sgemm_absprod(A, B, 1)
    assert componentwise_err(r, ref, ab) <= fp32_bound(80)


def test_dgemm_ld_oracle_accuracy():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((20, 30)) * 1e3
    B = rng.standard_normal((30, 10)) * 1e-3
    ref = orc.dgemm_ld(A, B, 0)
    assert normwise_err(ref, A @ B) < 1e-14


def test_normal_scaled_generator():
    x, s = orc.normal_scaled_f64(7, 10001)
    assert 1e-3 <= s <= 1e3
    z = x / s
    assert abs(z.mean()) < 0.05 and abs(z.std() - 1) < 0.05
    x2, s2 = orc.normal_scaled_f64(7, 10001)
    assert np.array_equal(x, x2) and s == s2


FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_fixture(path):
    """(kind, A, B, reference C) of a golden fixture; the inputs are
    regenerated from the stored seed with the reference benchmarks' generator."""
    f = np.load(path)
    kind = str(f["kind"])
    M, N, K, seed = (int(f[k]) for k in ("M", "N", "K", "seed"))
    if kind == "sgemm_nt_ref":
        A, B = orc.gemm_inputs_f32(seed, M, N, K, 1)
    elif kind in ("sgemm_nn_ref", "sgemm_mp_ngm_ref"):
        A, B = orc.gemm_inputs_f32(seed, M, N, K, 0)
    elif kind == "dgemm_nn_ref":
        A, B = orc.dgemm_inputs(seed, M, N, K)
    else:
        raise ValueError(kind)
    return kind, A, B, f["C"]


def test_fixtures_present():
    kinds = {str(np.load(p)["kind"]) for p in FIXTURES}
    assert kinds == {"sgemm_nt_ref", "sgemm_nn_ref", "dgemm_nn_ref", "sgemm_mp_ngm_ref"}
    assert any("sgemm_nt_80_seed0" in p for p in FIXTURES)  # LibShalom_sgemm(NoTrans, Trans), 80^3


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_golden_fixture_pins_restatement(path):
    """The fixtures hold the output of the reference's own instructions
    (tests/golden/make_golden.py).  The oracle's restatement of the reference's
    rounding order must reproduce every element the reference computes
    correctly, bit for bit."""
    kind, A, B, C = load_fixture(path)
    if kind == "sgemm_nt_ref":
        got = orc.sgemm_nt_reforder(A, B)
    elif kind == "sgemm_nn_ref":
        got = orc.sgemm_kseq(A, B, 0)
    elif kind == "sgemm_mp_ngm_ref":
        # GEMM_K = 320 blocked chains, block partials added into C in order;
        # every column outside the reference's defective 12-column edge
        ok = np.ones(C.shape[1], bool)
        ok[np.load(path)["edge_cols"]] = False
        assert not np.isnan(C).any()
        got = orc.sgemm_kseq(A, B, 0, kblock=320)
        assert np.array_equal(got[:, ok], C[:, ok])
        assert normwise_err(got, orc.sgemm_f64(A, B, 0)) <= 1e-6
        return
    else:
        got = orc.dgemm_reforder(A, B)
    assert got.shape == C.shape
    wrote = ~np.isnan(C)
    if kind != "dgemm_nn_ref":
        assert wrote.all()
        assert np.array_equal(got, C)
        return
    exact = orc.dgemm_ld(A, B, 0)
    correct = wrote & (np.abs(C - exact) <= 1e-12 * np.abs(exact).max())
    assert np.array_equal(got[correct], C[correct])
    # our restatement is the intended math everywhere, including where the
    # reference leaves C unwritten or wrong
    assert normwise_err(got, exact) <= 1e-14


def test_golden_dgemm_reference_defects_documented():
    """DGEMM_NN leaves the rows past 7*(M/7) unwritten when M % 7 is 1 or 4 and
    gets the N2-tail columns of the 2-row tail wrong; the fixtures record both."""
    bad = {os.path.basename(p): load_fixture(p) for p in FIXTURES
           if "dgemm_nn_22x16x5" in p or "dgemm_nn_23x26x13" in p}
    assert len(bad) == 2
    for name, (_, A, B, C) in bad.items():
        M, N = C.shape
        exact = orc.dgemm_ld(A, B, 0)
        body = slice(0, 7 * (M // 7))
        assert np.allclose(C[body][:, :6 * (N // 6)], exact[body][:, :6 * (N // 6)],
                           rtol=0, atol=1e-12 * np.abs(exact).max())
        tail = C[7 * (M // 7):]
        if M % 7 == 1:
            assert np.isnan(tail[:, :6 * (N // 6)]).all()   # never written
        else:
            wrong = np.abs(tail - exact[7 * (M // 7):]) > 1e-6 * np.abs(exact).max()
            assert wrong[:, 6 * (N // 6):].any()             # N2-tail values wrong
    with open(os.path.join(GOLDEN, "dgemm_reference_behaviour.json")) as fh:
        beh = json.load(fh)
    assert beh["M%7=1,N%6=2"]["unwritten_elements"] > 0
    assert beh["M%7=2,N%6=2"]["wrong_values"] > 0
    assert beh["M%7=6,N%6=1"]["wrong_values"] == 0


def test_golden_mp_reference_defect_documented():
    """The reference's NGM mp driver skips the K % 4 tail in its 12-column
    edge (the N == 12 packing path of SMM, NN_LIB/Kernel/SMM_m8n12_new.h,
    jumps past its RIGHT_K loop): with a K block that is not a multiple of 4
    those columns miss terms, far beyond FP32 rounding."""
    paths = [p for p in FIXTURES if "sgemm_mp_ngm" in p]
    defective = [p for p in paths if len(np.load(p)["edge_cols"])]
    assert len(defective) == 2 and len(paths) > len(defective)
    for p in defective:
        _, A, B, C = load_fixture(p)
        cols = np.load(p)["edge_cols"]
        exact = orc.sgemm_f64(A, B, 0)
        bound = fp32_bound(A.shape[1]) * orc.sgemm_absprod(A, B, 0)
        assert (np.abs(C[:, cols] - exact[:, cols]) > 10 * bound[:, cols]).any()
