"""GPU parity of LibShalom_dgemm_batched on the tensor cores (FP64 DMMA and
the Ozaki INT8-slice emulation), through the C ABI.

Tolerance: normwise max|C - C_ref| / max|C_ref| <= 1e-14 per C block, C_ref
from the extended-precision FP64 oracle applied product by product
(C = alpha_p A_p op(B_p) + beta_p C)."""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import normwise_err, to_dev, to_host
from tests.test_gpu_plain import _dgemm_runs, run_errors

pytestmark = pytest.mark.gpu

TOL = 1e-14
METHODS = [(ls.DGEMM_DMMA, 0), (ls.DGEMM_OZAKI, 0)]  # Ozaki default: 9 slices
IDS = ["dmma", "ozaki"]


@pytest.fixture
def method_reset():
    yield
    ls.set_dgemm_method(ls.DGEMM_FMA, 0)


@pytest.mark.parametrize("method,slices", METHODS + [(ls.DGEMM_OZAKI, 8)], ids=IDS + ["ozaki8"])
def test_runs_of_8_config_sizes(method, slices, method_reset):
    """the batched-DGEMM workload: runs of 8 products share C, sizes from
    {5,9,13,16,22,23,26,32}, entries normal(0,1) * 10^u per matrix"""
    dE, dC, ref, count, blocks = _dgemm_runs(300, 8, [5, 9, 13, 16, 22, 23, 26, 32], 11)
    ls.set_dgemm_method(method, slices)
    ls.dgemm_batched(dE, count)
    assert max(run_errors(to_host(dC), ref, blocks)) <= TOL


def _general(runs, seed):
    """Runs with explicit layouts.  runs: list of (M, N, ldc, c_nan, products)
    with products a list of (K, transb, alpha, beta, lda_pad, ldb_pad, odd):
    odd shifts A and B by one double (8-byte aligned operands)."""
    import torch
    _, ddt = ls.entry_dtypes()
    rng = np.random.default_rng(seed)
    flatA, flatB, flatC = [], [], []
    oa = ob = oc = 0
    recs = []
    for (M, N, ldc, c_nan, prods) in runs:
        C0 = rng.standard_normal((M, ldc))
        if c_nan:
            C0[:, :N] = np.nan
        flatC.append(C0.ravel())
        crec = (oc, M, N, ldc, C0.copy())
        oc += M * ldc
        plist = []
        for (K, tb, alpha, beta, lpa, lpb, odd) in prods:
            lda = K + lpa
            ldb = (K if tb else N) + lpb
            rows_b = N if tb else K
            pa = np.zeros(odd + M * lda)
            pb = np.zeros(odd + rows_b * ldb)
            A = rng.standard_normal((M, K)) * 10.0 ** rng.uniform(-2, 2)
            B = rng.standard_normal((rows_b, N if not tb else K)) * 10.0 ** rng.uniform(-2, 2)
            if M * lda:
                pa[odd:].reshape(M, lda)[:, :K] = A
            if rows_b * ldb:
                pb[odd:].reshape(rows_b, ldb)[:, :B.shape[1]] = B
            flatA.append(pa)
            flatB.append(pb)
            plist.append((oa + odd, ob + odd, M, N, K, tb, lda, ldb, alpha, beta, A, B))
            oa += len(pa)
            ob += len(pb)
        recs.append((crec, plist))
    dA = to_dev(np.concatenate(flatA + [np.zeros(2)]))
    dB = to_dev(np.concatenate(flatB + [np.zeros(2)]))
    dC = to_dev(np.concatenate(flatC))
    ent = []
    refs = []
    for (crec, plist) in recs:
        (o, M, N, ldc, C0) = crec
        C = C0[:, :N].copy()
        for (a0, b0, M_, N_, K, tb, lda, ldb, alpha, beta, A, B) in plist:
            ent.append((dA.data_ptr() + 8 * a0, dB.data_ptr() + 8 * b0, dC.data_ptr() + 8 * o,
                        M_, N_, K, tb, lda, ldb, ldc, 0, alpha, beta))
            C = orc.dgemm_ld(A, B, tb, alpha=alpha, beta=beta, C=C)
        refs.append((o, M, N, ldc, C0, C))
    arr = np.array(ent, ddt)
    dE = torch.from_numpy(arr.view(np.uint8)).cuda()
    return dE, len(arr), dC, refs


GENERAL = [
    # 32 x 32 block, K over several pieces, transposes, alpha/beta, padding, odd offsets
    (32, 32, 35, False, [(70, 1, -0.5, 2.0, 3, 1, 1), (33, 0, 1.0, 1.0, 0, 2, 0),
                         (32, 1, 1.5, -1.0, 1, 0, 1)]),
    # 1 x 1 with K = 1, K = 0 (beta only) and K = 33
    (1, 1, 1, False, [(1, 0, 1.0, 1.0, 0, 0, 0), (0, 0, 1.0, 0.5, 0, 0, 0),
                      (33, 1, 1.0, 1.0, 0, 0, 1)]),
    # first product with beta = 0 over a C of NaNs
    (13, 5, 6, True, [(9, 0, 1.0, 0.0, 0, 0, 1), (22, 1, 1.0, 1.0, 2, 0, 0)]),
    # a run longer than one warp's entry batch (40 products)
    (7, 29, 29, False, [(int(k), int(t), 1.0, 1.0, 0, 0, int(o))
                        for k, t, o in zip(np.arange(40) % 37 + 1, np.arange(40) % 2,
                                           np.arange(40) % 3 == 0)]),
    # blocks above 32 x 32 take the CUDA-core kernel
    (40, 20, 20, False, [(16, 0, 1.0, 1.0, 0, 0, 0), (5, 1, 2.0, 1.0, 0, 0, 1)]),
    (20, 33, 33, False, [(12, 0, 1.0, 1.0, 0, 0, 0)]),
]


@pytest.mark.parametrize("method,slices", METHODS, ids=IDS)
def test_general_layouts(method, slices, method_reset):
    dE, count, dC, refs = _general(GENERAL, 3)
    ls.set_dgemm_method(method, slices)
    ls.dgemm_batched(dE, count)
    got = to_host(dC)
    for (o, M, N, ldc, C0, C) in refs:
        blk = got[o:o + M * ldc].reshape(M, ldc)
        assert np.isfinite(blk[:, :N]).all(), (M, N)
        assert normwise_err(blk[:, :N], C) <= TOL, (M, N)
        # the padding columns of C are left alone
        assert np.array_equal(blk[:, N:], C0[:, N:]), (M, N)


@pytest.mark.parametrize("method,slices", METHODS, ids=IDS)
def test_many_runs_per_warp(method, slices, method_reset):
    """more runs than warps: every warp walks several runs (C-block reload,
    slot and ring reuse across runs)"""
    dE, dC, ref, count, blocks = _dgemm_runs(3000, 3, [1, 2, 5, 8, 17, 32], 5)
    ls.set_dgemm_method(method, slices)
    ls.dgemm_batched(dE, count)
    assert max(run_errors(to_host(dC), ref, blocks)) <= TOL


def test_method_setter_rejects_bad_values(method_reset):
    assert ls.lib().LibShalom_set_dgemm_method(7, 0) == ls.ERR_INVALID_VALUE
    assert ls.lib().LibShalom_set_dgemm_method(ls.DGEMM_OZAKI, 3) == ls.ERR_INVALID_VALUE
    assert ls.lib().LibShalom_set_dgemm_method(ls.DGEMM_OZAKI, 10) == ls.ERR_INVALID_VALUE
    ls.set_dgemm_method(ls.DGEMM_DMMA, 0)
    assert ls.get_dgemm_method() == ls.DGEMM_DMMA


@pytest.mark.parametrize("slices", [5, 6, 7])
def test_ozaki_error_shrinks_with_slices(slices, method_reset):
    """fewer digits: a larger but still bounded error, about 2^(-7S) relative"""
    dE, dC, ref, count, blocks = _dgemm_runs(200, 8, [5, 9, 13, 16, 22, 23, 26, 32], 17)
    ls.set_dgemm_method(ls.DGEMM_OZAKI, slices)
    ls.dgemm_batched(dE, count)
    err = max(run_errors(to_host(dC), ref, blocks))
    assert err <= 2.0 ** (-7 * slices) * 2000, err


@pytest.mark.parametrize("transb", [0, 1], ids=["nn", "nt"])
def test_fma_runs_bitexact_with_kseq_oracle(transb, method_reset):
    """The FP64 FMA grouped kernel (LIBSHALOM_DGEMM_FMA) with alpha = 1, beta =
    0 and one product per C: every element is one fused multiply-add chain
    over k in increasing order, bit for bit the oracle's k-sequential
    restatement, across single and multi-tile blocks, K below, at and above
    one 32-k slab, and every residue of M and N modulo the 4 x 4 thread
    tile."""
    import torch
    shapes = [(5, 13, 1), (13, 5, 7), (32, 32, 31), (32, 32, 32), (33, 40, 33), (40, 33, 70),
              (6, 7, 64), (17, 30, 95)]
    rng = np.random.default_rng(4242 + transb)
    _, ddt = ls.entry_dtypes()
    ent = np.zeros(len(shapes), ddt)
    As, Bs, offs = [], [], []
    oa = ob = oc = 0
    for i, (M, N, K) in enumerate(shapes):
        A = rng.standard_normal((M, K))
        B = rng.standard_normal((N, K) if transb else (K, N))
        As.append(A.ravel())
        Bs.append(B.ravel())
        offs.append((oa, ob, oc))
        oa += A.size
        ob += B.size
        oc += M * N
    dA = to_dev(np.concatenate(As))
    dB = to_dev(np.concatenate(Bs))
    dC = torch.full((oc,), float("nan"), dtype=torch.float64, device="cuda")
    for i, (M, N, K) in enumerate(shapes):
        a0, b0, c0 = offs[i]
        ent[i]["A"] = dA.data_ptr() + 8 * a0
        ent[i]["B"] = dB.data_ptr() + 8 * b0
        ent[i]["C"] = dC.data_ptr() + 8 * c0
        ent[i]["M"], ent[i]["N"], ent[i]["K"], ent[i]["transb"] = M, N, K, transb
        ent[i]["alpha"], ent[i]["beta"] = 1.0, 0.0
    dE = torch.from_numpy(ent.view(np.uint8)).cuda()
    ls.set_dgemm_method(ls.DGEMM_FMA, 0)
    ls.dgemm_batched(dE, len(shapes))
    got = to_host(dC)
    for i, (M, N, K) in enumerate(shapes):
        a0, b0, c0 = offs[i]
        A = As[i].reshape(M, K)
        B = Bs[i].reshape((N, K) if transb else (K, N))
        ref = orc.dgemm_kseq(A, B, transb)
        assert np.array_equal(got[c0:c0 + M * N].reshape(M, N), ref), (M, N, K)
