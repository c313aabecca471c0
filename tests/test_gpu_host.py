"""GPU parity of the host-memory calls (operands in host memory, as in the
reference's own API), through the C ABI.

The host calls run the same kernels as the device-pointer calls on staged
copies, so their results are compared BIT-EXACTLY with the device-pointer
calls and with the oracle's k-sequential restatement (plain paths), and with
the FP64 / long-double oracle under the tolerances of the device paths:
normwise max|C - C_ref| / max|C_ref| <= 1e-6 (FP32 and split-BF16 x6),
<= 1e-14 (FP64)."""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import normwise_err, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture
def reset():
    yield
    ls.set_precision(ls.PREC_FP32)
    ls.set_sync(True)
    ls.set_stream(None)


def test_sgemm_host_config1_bitexact():
    # LibShalom_sgemm(NoTrans, Trans) at 80^3 on host arrays
    A, B = orc.gemm_inputs_f32(0, 80, 80, 80, 1)
    C = np.full((80, 80), np.nan, dtype=np.float32)
    ls.sgemm_host(ls.NoTrans, ls.Trans, C, A, B, 80, 80, 80)
    assert np.array_equal(C, orc.sgemm_kseq(A, B, 1))


@pytest.mark.parametrize("transb", [0, 1])
def test_sgemm_host_tails_bitexact(transb):
    for (M, N, K) in [(1, 1, 1), (5, 16, 8), (17, 13, 15), (96, 33, 7)]:
        A, B = orc.gemm_inputs_f32(M + N + K, M, N, K, transb)
        C = np.empty((M, N), dtype=np.float32)
        ls.sgemm_host(0, transb, C, A, B, M, N, K)
        assert np.array_equal(C, orc.sgemm_kseq(A, B, transb)), (M, N, K)


@pytest.mark.parametrize("prec", [ls.PREC_FP32, ls.PREC_BF16X6])
@pytest.mark.parametrize("M,N,K", [(256, 196, 2304), (64, 3136, 576)])
def test_sgemm_mp_host_matches_device(prec, M, N, K, reset):
    import torch
    A, B = orc.gemm_inputs_f32(M * 3 + N, M, N, K, 0)
    ls.set_precision(prec)
    C = np.full((M, N), np.nan, dtype=np.float32)
    ls.sgemm_mp_host(0, 0, C, A, B, M, N, K)
    dC = torch.full((M, N), float("nan"), device="cuda")
    ls.sgemm_mp(0, 0, dC, to_dev(A), to_dev(B), M, N, K)
    assert np.array_equal(C, to_host(dC))
    assert normwise_err(C, orc.sgemm_f64(A, B, 0)) <= 1e-6


def test_dgemm_host_config_sizes():
    rng = np.random.default_rng(5)
    for M in (5, 13, 22, 32):
        for K in (9, 26):
            N = 23
            A = rng.standard_normal((M, K)) * 10.0 ** rng.uniform(-3, 3)
            B = rng.standard_normal((K, N))
            C = np.empty((M, N))
            ls.dgemm_host(0, 0, C, A, B, M, N, K)
            assert np.array_equal(C, orc.dgemm_kseq(A, B, 0)), (M, K)
            assert normwise_err(C, orc.dgemm_ld(A, B, 0)) <= 1e-14


def test_host_call_rejects_bad_arguments():
    A = np.zeros(16, np.float32)
    st = ls.sgemm_host(2, 0, A, A, A, 4, 4, 1, check=False)
    assert st == ls.ERR_INVALID_VALUE
    # overlapping outputs cannot be copied back
    st = ls.sgemm_batched_strided_host(0, 2, 2, 2, 1.0, A, 4, A, 4, 0.0, A, 3, 2, check=False)
    assert st == ls.ERR_INVALID_VALUE


def _batch(rng, count, M, N, K, tb, sA, sB, sC):
    A = rng.uniform(-1, 1, size=count * sA + M * K).astype(np.float32)
    B = rng.uniform(-1, 1, size=count * sB + K * N).astype(np.float32)
    C = rng.uniform(-1, 1, size=count * sC + M * N).astype(np.float32)
    return A, B, C


def _ref(A, B, C0, g, M, N, K, tb, sA, sB, sC, alpha, beta):
    a = A[g * sA:g * sA + M * K].reshape(M, K)
    b = B[g * sB:g * sB + K * N].reshape((N, K) if tb else (K, N))
    c = C0[g * sC:g * sC + M * N].reshape(M, N)
    return orc.sgemm_f64(a, b, tb, alpha=alpha, beta=beta, C=c)


@pytest.mark.parametrize("prec", [ls.PREC_FP32, ls.PREC_BF16X6])
@pytest.mark.parametrize("tb", [0, 1])
def test_batched_host_many_chunks_matches_device(prec, tb, reset):
    """1,000 GEMMs of 128^3 (three 64 MB chunks), pinned host memory, async
    mode on a side stream: identical to the device-pointer call."""
    import torch
    n, count = 128, 1000
    ls.set_precision(prec)
    g = torch.Generator().manual_seed(11 + tb)
    hA = (torch.rand(count * n * n, generator=g) * 2 - 1).pin_memory()
    hB = (torch.rand(count * n * n, generator=g) * 2 - 1).pin_memory()
    hC = torch.full((count * n * n,), float("nan")).pin_memory()
    s = torch.cuda.Stream()
    ls.set_stream(s)
    ls.set_sync(False)
    ls.sgemm_batched_strided_host(tb, n, n, n, 1.0, hA, n * n, hB, n * n, 0.0, hC, n * n, count)
    ls.synchronize()
    ls.set_sync(True)
    ls.set_stream(None)  # the device-pointer call below follows torch's copies
    dC = torch.empty(count * n * n, device="cuda")
    ls.sgemm_batched_strided(tb, n, n, n, 1.0, hA.cuda(), n * n, hB.cuda(), n * n, 0.0, dC,
                             n * n, count)
    torch.cuda.synchronize()
    assert torch.equal(hC, dC.cpu())
    A, B, C = hA.numpy(), hB.numpy(), hC.numpy()
    for gi in (0, 340, 341, 999):  # both sides of the first chunk boundary (341 per chunk)
        ref = _ref(A, B, C, gi, n, n, n, tb, n * n, n * n, n * n, 1.0, 0.0)
        got = C[gi * n * n:(gi + 1) * n * n].reshape(n, n)
        assert normwise_err(got, ref) <= 1e-6, gi


@pytest.mark.parametrize("prec", [ls.PREC_FP32, ls.PREC_BF16X6])
def test_batched_host_gaps_beta_and_broadcast(prec, reset):
    """Pageable numpy arrays; A and C with gaps between matrices, B shared by
    every GEMM (stride 0), beta != 0 (C copied in); the gaps stay untouched."""
    rng = np.random.default_rng(9)
    M, N, K, count, tb = 37, 53, 71, 300, 0
    sA, sB, sC = M * K + 5, 0, M * N + 3
    A, B, C0 = _batch(rng, count, M, N, K, tb, sA, sB, sC)
    C = C0.copy()
    ls.set_precision(prec)
    ls.sgemm_batched_strided_host(tb, M, N, K, -0.5, A, sA, B, sB, 1.25, C, sC, count)
    for gi in (0, 1, 150, 299):
        ref = _ref(A, B, C0, gi, M, N, K, tb, sA, sB, sC, -0.5, 1.25)
        got = C[gi * sC:gi * sC + M * N].reshape(M, N)
        assert normwise_err(got, ref) <= 1e-6, gi
    mask = np.ones(C.size, bool)
    for gi in range(count):
        mask[gi * sC:gi * sC + M * N] = False
    assert np.array_equal(C[mask], C0[mask])
