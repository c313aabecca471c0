"""GPU parity of the split-BF16 tensor-core path (tcgen05), through the C ABI.

Floating-point tolerance (stated per mode, against the exact-math oracle):
  bf16x6 (hi/mid/lo, 6 products): normwise max|C - C64| / max|C64| <= 1e-6
  bf16x3 (hi/lo, 3 products):     normwise <= 2e-5
and componentwise |C - C64|_ij <= tol_c * (|A||B|)_ij with tol_c = 8 * 2^-24
(bf16x6) or 2^-14 (bf16x3)."""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import componentwise_err, normwise_err, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL = {ls.PREC_BF16X6: (1e-6, 8 * 2.0 ** -24), ls.PREC_BF16X3: (2e-5, 2.0 ** -14)}


@pytest.fixture
def mode_setter():
    yield ls.set_precision
    ls.set_precision(ls.PREC_FP32)
    ls.set_tma(True)


@pytest.fixture(params=[True, False], ids=["tma", "cpasync"])
def staging(request):
    """both operand-staging variants of the tensor-core kernel"""
    ls.set_tma(request.param)
    yield request.param
    ls.set_tma(True)


def _strided(mode, transb, M, N, K, count, seed, alpha=1.0, beta=0.0):
    import torch
    A = orc.uniform_f32(seed, count * M * K).reshape(count, M, K)
    B = orc.uniform_f32(seed + 1, count * K * N).reshape((count, N, K) if transb
                                                         else (count, K, N))
    C0 = orc.uniform_f32(seed + 2, count * M * N).reshape(count, M, N)
    dC = to_dev(C0) if beta != 0.0 else torch.full((count, M, N), float("nan"),
                                                     device="cuda")
    ls.set_precision(mode)
    ls.sgemm_batched_strided(transb, M, N, K, alpha, to_dev(A), M * K, to_dev(B), K * N, beta,
                             dC, M * N, count)
    return A, B, C0, to_host(dC)


def _check(C, A, B, transb, mode, alpha=1.0, beta=0.0, C0=None):
    ref = orc.sgemm_f64(A, B, transb, alpha=alpha, beta=beta, C=C0)
    nw, cw = TOL[mode]
    e = normwise_err(C, ref)
    assert e <= nw, e
    if beta == 0.0:
        assert componentwise_err(C, ref, abs(alpha) * orc.sgemm_absprod(A, B, transb)) <= cw
    return e


@pytest.mark.parametrize("mode", [ls.PREC_BF16X6, ls.PREC_BF16X3])
@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("n", list(range(8, 129, 8)))
def test_tc_cube_sweep(n, transb, mode, mode_setter, staging):
    count = 37
    A, B, _, C = _strided(mode, transb, n, n, n, count, seed=100 + n + 7 * transb)
    for g in (0, 1, count // 2, count - 1):
        _check(C[g], A[g], B[g], transb, mode)


@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (3, 5, 7), (13, 9, 33), (17, 31, 15),
                                   (64, 64, 64), (65, 17, 40), (100, 130, 70),
                                   (129, 7, 200), (33, 129, 31), (200, 250, 257)])
def test_tc_ragged(M, N, K, transb, mode_setter, staging):
    count = 9
    A, B, _, C = _strided(ls.PREC_BF16X6, transb, M, N, K, count, seed=M * 7 + N * 3 + K)
    for g in range(count):
        _check(C[g], A[g], B[g], transb, ls.PREC_BF16X6)


def test_tc_alpha_beta(mode_setter):
    A, B, C0, C = _strided(ls.PREC_BF16X6, 1, 24, 40, 56, 20, seed=5, alpha=-0.5, beta=1.0)
    for g in range(20):
        _check(C[g], A[g], B[g], 1, ls.PREC_BF16X6, alpha=-0.5, beta=1.0, C0=C0[g])


@pytest.mark.parametrize("M,N,K", [(64, 392, 576), (128, 98, 1152), (512, 49, 960),
                                   (2048, 32, 2560), (32, 2048, 1024)])
def test_tc_sgemm_mp(M, N, K, mode_setter, staging):
    import torch
    A, B = orc.gemm_inputs_f32(M + 2 * N + K, M, N, K, 0)
    dC = torch.full((M, N), float("nan"), device="cuda")
    ls.set_precision(ls.PREC_BF16X6)
    ls.sgemm_mp(0, 0, dC, to_dev(A), to_dev(B), M, N, K)
    _check(to_host(dC), A, B, 0, ls.PREC_BF16X6)


def test_tc_large_batch_spot_check(mode_setter, staging):
    # many tiles per CTA: the persistent loop, buffer/phase reuse across tiles
    count, n = 3000, 40
    A, B, _, C = _strided(ls.PREC_BF16X6, 0, n, n, n, count, seed=9)
    for g in (0, 1, 2, 1499, 2998, 2999):
        _check(C[g], A[g], B[g], 0, ls.PREC_BF16X6)
