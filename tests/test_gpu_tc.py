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


@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("M,N,K", [(8, 8, 8), (12, 20, 24), (24, 24, 24), (20, 60, 33),
                                   (40, 40, 40), (56, 56, 56), (64, 64, 64), (60, 64, 17),
                                   (16, 52, 70), (13, 9, 33), (72, 72, 72), (130, 100, 64)])
def test_tc_batch_every_gemm_and_nothing_past_c(M, N, K, transb, mode_setter):
    """Every GEMM of a batch whose count leaves a partial last tile (packed
    small GEMMs with row stores; one GEMM per tile with C by TMA boxes), and
    the floats after the batch's C stay as they were."""
    import torch
    count = 53
    A = orc.uniform_f32(M + N + K, count * M * K).reshape(count, M, K)
    B = orc.uniform_f32(M + N + K + 1, count * K * N).reshape((count, N, K) if transb
                                                              else (count, K, N))
    buf = torch.full((count * M * N + 256,), 7.0, device="cuda")
    ls.set_precision(ls.PREC_BF16X6)
    ls.sgemm_batched_strided(transb, M, N, K, 1.0, to_dev(A), M * K, to_dev(B), K * N, 0.0,
                             buf, M * N, count)
    h = to_host(buf)
    assert np.all(h[count * M * N:] == 7.0)
    C = h[:count * M * N].reshape(count, M, N)
    for g in range(count):
        _check(C[g], A[g], B[g], transb, ls.PREC_BF16X6)


@pytest.mark.parametrize("mode", [ls.PREC_BF16X6, ls.PREC_BF16X3])
@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("M,N,K", [(100, 1, 40), (130, 16, 33), (96, 17, 300), (200, 32, 64),
                                   (70, 29, 700), (96, 48, 520), (130, 64, 300), (70, 65, 300)])
def test_tc_narrow_tiles(M, N, K, transb, mode, mode_setter, staging):
    """Tiles of at most 32 columns, one GEMM per tile (MMA N of 16 or 32),
    short K and the long-K register fold; with long K, tiles of 48 and 64
    columns take the narrow fold (one 32-column block per epilogue warp) and
    80 columns the full one."""
    count = 5
    A, B, _, C = _strided(mode, transb, M, N, K, count, seed=M + 3 * N + K + transb)
    for g in range(count):
        _check(C[g], A[g], B[g], transb, mode)


@pytest.mark.parametrize("mode", [ls.PREC_BF16X6, ls.PREC_BF16X3])
@pytest.mark.parametrize("splits", [0, 1, 5])
def test_tc_narrow_mp_long_k(splits, mode, mode_setter):
    """A tall, 32-column GEMM with long K (the 20480 x 32 x 20480 shape family)
    through sgemm_mp, with and without split-K."""
    import torch
    M, N, K = 1536, 32, 4160
    A, B = orc.gemm_inputs_f32(M + N + K + splits, M, N, K, 0)
    dC = torch.full((M, N), float("nan"), device="cuda")
    ls.set_precision(mode)
    ls.set_splitk(splits)
    try:
        ls.sgemm_mp(0, 0, dC, to_dev(A), to_dev(B), M, N, K)
    finally:
        ls.set_splitk(0)
    _check(to_host(dC), A, B, 0, mode)


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


# ---------------------------------------------------------------------------
# grouped batches (LibShalom_sgemm_batched) on the tensor cores
# ---------------------------------------------------------------------------
from tests.test_gpu_plain import _sgemm_entries, _split  # noqa: E402


@pytest.mark.parametrize("mode", [ls.PREC_BF16X6, ls.PREC_BF16X3])
def test_tc_grouped_mixed_log_uniform(mode, mode_setter):
    rng = np.random.default_rng(21)
    shapes = []
    for _ in range(400):
        M, N, K = (int(np.exp(rng.uniform(np.log(4), np.log(256)))) for _ in range(3))
        shapes.append((M, N, K, int(rng.integers(2))))
    b = _sgemm_entries(shapes, beta_choices=(0.0, 1.0))
    ls.set_precision(mode)
    ls.sgemm_batched(b["dE"], len(shapes))
    Cs = _split(to_host(b["dC"]), shapes)
    for i, (M, N, K, tb) in enumerate(shapes):
        ref = orc.sgemm_f64(b["As"][i], b["Bs"][i], tb, beta=b["betas"][i], C=b["C0s"][i])
        assert normwise_err(Cs[i], ref) <= TOL[mode][0], (i, M, N, K, tb)


def test_tc_grouped_large_and_long_k(mode_setter):
    shapes = [(300, 200, 700, 0), (130, 257, 129, 1), (5, 300, 1000, 0), (256, 256, 256, 1),
              (1, 1, 1, 0), (7, 3, 2000, 1)]
    b = _sgemm_entries(shapes, beta_choices=(1.0,))
    ls.set_precision(ls.PREC_BF16X6)
    ls.sgemm_batched(b["dE"], len(shapes))
    Cs = _split(to_host(b["dC"]), shapes)
    for i, (M, N, K, tb) in enumerate(shapes):
        ref = orc.sgemm_f64(b["As"][i], b["Bs"][i], tb, beta=1.0, C=b["C0s"][i])
        assert normwise_err(Cs[i], ref) <= 1e-6, (i, M, N, K)


def test_tc_grouped_runs_share_c(mode_setter):
    """consecutive entries naming the same C are applied in order (C += A_p B_p)"""
    import torch
    sdt, _ = ls.entry_dtypes()
    rng = np.random.default_rng(4)
    runs = [(24, 40, [16, 33, 7]), (130, 20, [64, 64]), (9, 9, [5] * 8)]
    As, Bs, C0 = [], [], []
    for (M, N, Ks) in runs:
        C0.append(orc.uniform_f32(len(C0) + 50, M * N))
        for K in Ks:
            As.append(orc.uniform_f32(len(As) + 100, M * K))
            Bs.append(orc.uniform_f32(len(Bs) + 200, K * N))
    dA = to_dev(np.concatenate(As))
    dB = to_dev(np.concatenate(Bs))
    dC = to_dev(np.concatenate(C0))
    ent, oa, ob, oc, p = [], 0, 0, 0, 0
    for (M, N, Ks) in runs:
        for K in Ks:
            ent.append((dA.data_ptr() + 4 * oa, dB.data_ptr() + 4 * ob, dC.data_ptr() + 4 * oc,
                        M, N, K, 0, 0, 0, 0, 1.0, 1.0, 0))
            oa += M * K
            ob += K * N
            p += 1
        oc += M * N
    arr = np.array(ent, sdt)
    ls.set_precision(ls.PREC_BF16X6)
    ls.sgemm_batched(torch.from_numpy(arr.view(np.uint8)).cuda(), len(arr))
    got = to_host(dC)
    oc, p = 0, 0
    for r, (M, N, Ks) in enumerate(runs):
        ref = C0[r].reshape(M, N).astype(np.float64)
        for K in Ks:
            ref = ref + As[p].reshape(M, K).astype(np.float64) @ Bs[p].reshape(K, N).astype(np.float64)
            p += 1
        assert normwise_err(got[oc:oc + M * N].reshape(M, N), ref) <= 1e-6, r
        oc += M * N


def test_tc_grouped_unaligned_leading_dims(mode_setter):
    import torch
    sdt, _ = ls.entry_dtypes()
    M, N, K = 37, 29, 45
    lda, ldb, ldc = 47, 31, 33   # not multiples of 4: the 4-byte copy path
    A = orc.uniform_f32(1, M * lda).reshape(M, lda)
    B = orc.uniform_f32(2, K * ldb).reshape(K, ldb)
    C = np.zeros((M, ldc), np.float32)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    arr = np.array([(dA.data_ptr() + 4, dB.data_ptr(), dC.data_ptr(), M, N, K, 0, lda, ldb, ldc,
                     1.0, 0.0, 0)], sdt)
    ls.set_precision(ls.PREC_BF16X6)
    ls.sgemm_batched(torch.from_numpy(arr.view(np.uint8)).cuda(), 1)
    got = to_host(dC)[:, :N]
    ref = orc.sgemm_f64(A[:, 1:1 + K], B[:, :N], 0)
    assert normwise_err(got, ref) <= 1e-6


def test_tc_grouped_even_leading_dims(mode_setter):
    """leading dimensions that are even but not multiples of 4 (8-byte copies),
    NN and NT"""
    import torch
    sdt, _ = ls.entry_dtypes()
    M, N, K = 70, 50, 90
    lda, ldc = 94, 58
    for tb in (0, 1):
        ldb = 98 if tb else 54  # >= K for B[N x K], >= N for B[K x N]
        A = orc.uniform_f32(3 + tb, M * lda).reshape(M, lda)
        B = orc.uniform_f32(5 + tb, (N if tb else K) * ldb).reshape(N if tb else K, ldb)
        C = np.zeros((M, ldc), np.float32)
        dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
        arr = np.array([(dA.data_ptr() + 8, dB.data_ptr(), dC.data_ptr(), M, N, K, tb, lda, ldb,
                         ldc, 1.0, 0.0, 0)], sdt)
        ls.set_precision(ls.PREC_BF16X6)
        ls.sgemm_batched(torch.from_numpy(arr.view(np.uint8)).cuda(), 1)
        got = to_host(dC)[:, :N]
        Bm = B[:, :K] if tb else B[:, :N]
        ref = orc.sgemm_f64(np.ascontiguousarray(A[:, 2:2 + K]), np.ascontiguousarray(Bm), tb)
        assert normwise_err(got, ref) <= 1e-6, tb


def test_tc_grouped_small_after_large_is_exact(mode_setter):
    """a CTA that runs a full 128x128 tile with non-finite operands and then a
    tiny GEMM: rows and columns the tiny GEMM does not stage must not reach
    its output"""
    import torch
    sdt, _ = ls.entry_dtypes()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    big, small = (128, 128, 96), (5, 7, 3)
    nb = sms
    Ab = orc.uniform_f32(11, big[0] * big[2])
    Ab[::17] = np.inf
    Bb = orc.uniform_f32(12, big[2] * big[1])
    Bb[::13] = np.nan
    As = orc.uniform_f32(13, small[0] * small[2])
    Bs = orc.uniform_f32(14, small[2] * small[1])
    dAb, dBb, dAs, dBs = to_dev(Ab), to_dev(Bb), to_dev(As), to_dev(Bs)
    dCb = torch.zeros(nb * big[0] * big[1], device="cuda")
    dCs = torch.full((nb * small[0] * small[1],), float("nan"), device="cuda")
    ent = []
    for i in range(nb):  # heavy runs first: one per CTA, then one light run per CTA
        ent.append((dAb.data_ptr(), dBb.data_ptr(), dCb.data_ptr() + 4 * i * big[0] * big[1],
                    big[0], big[1], big[2], 0, 0, 0, 0, 1.0, 0.0, 0))
    for i in range(nb):
        ent.append((dAs.data_ptr(), dBs.data_ptr(), dCs.data_ptr() + 4 * i * small[0] * small[1],
                    small[0], small[1], small[2], i & 1, 0, 0, 0, 1.0, 0.0, 0))
    arr = np.array(ent, sdt)
    ls.set_precision(ls.PREC_BF16X6)
    ls.sgemm_batched(torch.from_numpy(arr.view(np.uint8)).cuda(), len(arr))
    got = to_host(dCs).reshape(nb, small[0], small[1])
    for i in range(nb):
        tb = i & 1
        Bm = Bs.reshape(small[1], small[2]) if tb else Bs.reshape(small[2], small[1])
        ref = orc.sgemm_f64(As.reshape(small[0], small[2]), Bm, tb)
        assert np.isfinite(got[i]).all(), i
        assert normwise_err(got[i], ref) <= 1e-6, i


@pytest.mark.parametrize("splits", [0, 3, 8])
def test_tc_sgemm_mp_split_k(splits, mode_setter):
    """K slices of one GEMM as a batch of partial products plus an ordered
    reduction (auto choice, and forced factors that must divide K / 32)"""
    import torch
    M, N, K = 256, 196, 2304
    A, B = orc.gemm_inputs_f32(99, M, N, K, 0)
    dC = torch.full((M, N), float("nan"), device="cuda")
    ls.set_precision(ls.PREC_BF16X6)
    ls.set_splitk(splits)
    try:
        ls.sgemm_mp(0, 0, dC, to_dev(A), to_dev(B), M, N, K)
    finally:
        ls.set_splitk(0)
    _check(to_host(dC), A, B, 0, ls.PREC_BF16X6)
