"""GPU parity at the benchmark's full sizes, through the C ABI, checked
against the host oracle (oracle/oracle.c) on samples of every batch.

  mixed batch   50,000 GEMMs, M, N, K log-uniform integers in [4, 256],
                NN/NT 50/50, beta 0/1 (LibShalom_sgemm_batched), on every GEMM
                of the first 2,000 and 300 sampled later ones: split-BF16 x6
                within 8 u componentwise (u = 2^-24, relative to |A||B| +
                |beta C|) and 1e-6 normwise over the sample; plain FP32 within
                the deterministic bound gamma_(K+2) componentwise
  DGEMM runs    200,000 products, runs of 8 share C, sizes {5,...,32},
                entries normal(0,1) 10^u (LibShalom_dgemm_batched): FP64 FMA,
                DMMA and Ozaki (9 slices) within 1e-14 normwise per C block on
                300 sampled runs (extended-precision oracle over the run)
  uniform       10,000 GEMMs per size at n = 8, 64, 128, NN and NT
                (LibShalom_sgemm_batched_strided): plain FP32 bit-exact with the
                k-sequential restatement, split-BF16 x6 within 1e-6, on 64
                sampled GEMMs each
  irregular     the six LibShalom_sgemm_mp shapes incl. 20480 x 32 x 20480:
                plain FP32 without split-K bit-exact with the GEMM_K-blocked
                restatement, split-BF16 x6 within 1e-6, on 48 sampled rows
"""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import componentwise_err, fp32_bound, normwise_err, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture
def reset():
    yield
    ls.set_precision(ls.PREC_FP32)
    ls.set_dgemm_method(ls.DGEMM_FMA, 0)
    ls.set_splitk(0)


def _mixed(count, seed):
    rng = np.random.default_rng(seed)
    dims = np.exp(rng.uniform(np.log(4), np.log(256), size=(count, 3))).astype(np.int64)
    M, N, K = dims[:, 0], dims[:, 1], dims[:, 2]
    tb = rng.integers(2, size=count)
    beta = rng.integers(2, size=count).astype(np.float32)
    a_len, b_len, c_len = M * K, K * N, M * N
    offs = [np.concatenate([[0], np.cumsum(x)[:-1]]) for x in (a_len, b_len, c_len)]
    hA = rng.uniform(-1, 1, int(a_len.sum())).astype(np.float32)
    hB = rng.uniform(-1, 1, int(b_len.sum())).astype(np.float32)
    hC = rng.uniform(-1, 1, int(c_len.sum())).astype(np.float32)
    return M, N, K, tb, beta, offs, hA, hB, hC


def test_mixed_batch_50000(reset):
    import torch
    count = 50_000
    M, N, K, tb, beta, offs, hA, hB, hC = _mixed(count, 2024)
    dA, dB, dC = to_dev(hA), to_dev(hB), to_dev(hC)
    sdt, _ = ls.entry_dtypes()
    ent = np.zeros(count, sdt)
    ent["A"] = dA.data_ptr() + 4 * offs[0]
    ent["B"] = dB.data_ptr() + 4 * offs[1]
    ent["C"] = dC.data_ptr() + 4 * offs[2]
    ent["M"], ent["N"], ent["K"], ent["transb"] = M, N, K, tb
    ent["alpha"] = 1.0
    ent["beta"] = beta
    dE = torch.from_numpy(ent.view(np.uint8)).cuda()
    rng = np.random.default_rng(1)
    sample = np.concatenate([np.arange(2000), rng.choice(np.arange(2000, count), 300, False)])
    for prec in (ls.PREC_BF16X6, ls.PREC_FP32):
        dC.copy_(torch.from_numpy(hC))
        ls.set_precision(prec)
        ls.sgemm_batched(dE, count)
        got = to_host(dC)
        num = den = 0.0
        for i in sample:
            m, n, k = int(M[i]), int(N[i]), int(K[i])
            a = hA[offs[0][i]:offs[0][i] + m * k].reshape(m, k)
            bsrc = hB[offs[1][i]:offs[1][i] + k * n]
            b = bsrc.reshape(n, k) if tb[i] else bsrc.reshape(k, n)
            c0 = hC[offs[2][i]:offs[2][i] + m * n].reshape(m, n)
            ref = orc.sgemm_f64(a, b, int(tb[i]), beta=float(beta[i]), C=c0)
            c = got[offs[2][i]:offs[2][i] + m * n].reshape(m, n)
            scale = orc.sgemm_absprod(a, b, int(tb[i])) + abs(float(beta[i])) * np.abs(c0)
            bound = 8 * 2.0 ** -24 if prec == ls.PREC_BF16X6 else fp32_bound(k + 2)
            e = componentwise_err(c, ref, scale)
            assert e <= bound, (prec, i, m, n, k, int(tb[i]), float(beta[i]), e)
            num = max(num, float(np.max(np.abs(c - ref))))
            den = max(den, float(np.max(np.abs(ref))))
        if prec == ls.PREC_BF16X6:
            assert num / den <= 1e-6


def test_dgemm_runs_200000(reset):
    import torch
    count, run = 200_000, 8
    sizes = np.array([5, 9, 13, 16, 22, 23, 26, 32])
    rng = np.random.default_rng(77)
    nruns = count // run
    Mr = sizes[rng.integers(len(sizes), size=nruns)]
    Nr = sizes[rng.integers(len(sizes), size=nruns)]
    M, N = np.repeat(Mr, run), np.repeat(Nr, run)
    K = sizes[rng.integers(len(sizes), size=count)]
    a_len, b_len, c_len = M * K, K * N, Mr * Nr
    offA = np.concatenate([[0], np.cumsum(a_len)[:-1]])
    offB = np.concatenate([[0], np.cumsum(b_len)[:-1]])
    offCr = np.concatenate([[0], np.cumsum(c_len)[:-1]])
    offC = np.repeat(offCr, run)
    hA = rng.standard_normal(int(a_len.sum())) * np.repeat(10.0 ** rng.uniform(-3, 3, count), a_len)
    hB = rng.standard_normal(int(b_len.sum())) * np.repeat(10.0 ** rng.uniform(-3, 3, count), b_len)
    hC = rng.standard_normal(int(c_len.sum()))
    dA, dB, dC = to_dev(hA), to_dev(hB), to_dev(hC)
    _, ddt = ls.entry_dtypes()
    ent = np.zeros(count, ddt)
    ent["A"] = dA.data_ptr() + 8 * offA
    ent["B"] = dB.data_ptr() + 8 * offB
    ent["C"] = dC.data_ptr() + 8 * offC
    ent["M"], ent["N"], ent["K"] = M, N, K
    ent["alpha"] = 1.0
    ent["beta"] = 1.0
    dE = torch.from_numpy(ent.view(np.uint8)).cuda()
    samp = np.sort(rng.choice(nruns, 300, replace=False))
    # oracle of the sampled runs: C0 + the run's products in extended precision
    refs = {}
    i32 = lambda v: np.ascontiguousarray(v, np.int32)  # noqa: E731
    i64 = lambda v: np.ascontiguousarray(v, np.int64)  # noqa: E731
    for r in samp:
        sl = slice(r * run, (r + 1) * run)
        c = hC[offCr[r]:offCr[r] + c_len[r]].copy()
        orc.lib().orc_dgemm_batched_ld(run, i32(M[sl]), i32(N[sl]), i32(K[sl]), hA,
                                       i64(offA[sl]), hB, i64(offB[sl]), c,
                                       i64(offC[sl] - offCr[r]))
        refs[r] = c
    for meth, sl in ((ls.DGEMM_FMA, 0), (ls.DGEMM_DMMA, 0), (ls.DGEMM_OZAKI, 9)):
        dC.copy_(torch.from_numpy(hC))
        ls.set_dgemm_method(meth, sl)
        ls.dgemm_batched(dE, count)
        got = to_host(dC)
        for r in samp:
            e = normwise_err(got[offCr[r]:offCr[r] + c_len[r]], refs[r])
            assert e <= 1e-14, (meth, r, int(Mr[r]), int(Nr[r]), e)


@pytest.mark.parametrize("n", [8, 64, 128])
@pytest.mark.parametrize("tb", [0, 1], ids=["nn", "nt"])
def test_uniform_batch_10000(n, tb, reset):
    import torch
    count = 10_000
    rng = np.random.default_rng(n + 1000 * tb)
    hA = rng.uniform(-1, 1, count * n * n).astype(np.float32)
    hB = rng.uniform(-1, 1, count * n * n).astype(np.float32)
    dA, dB = to_dev(hA), to_dev(hB)
    dC = torch.full((count * n * n,), float("nan"), device="cuda")
    samp = np.concatenate([[0, count - 1], rng.choice(count, 62, replace=False)])
    for prec in (ls.PREC_FP32, ls.PREC_BF16X6):
        ls.set_precision(prec)
        ls.sgemm_batched_strided(tb, n, n, n, 1.0, dA, n * n, dB, n * n, 0.0, dC, n * n, count)
        got = to_host(dC).reshape(count, n, n)
        for g in samp:
            a = hA[g * n * n:(g + 1) * n * n].reshape(n, n)
            b = hB[g * n * n:(g + 1) * n * n].reshape(n, n)
            if prec == ls.PREC_FP32:
                assert np.array_equal(got[g], orc.sgemm_kseq(a, b, tb)), (n, tb, g)
            else:
                assert normwise_err(got[g], orc.sgemm_f64(a, b, tb)) <= 1e-6, (n, tb, g)


IRREGULAR = [(64, 3136, 576), (128, 784, 1152), (256, 196, 2304), (512, 49, 4608),
             (20480, 32, 20480), (32, 20480, 4096)]


@pytest.mark.parametrize("M,N,K", IRREGULAR, ids=[f"{m}x{n}x{k}" for m, n, k in IRREGULAR])
def test_irregular_shape(M, N, K, reset):
    import torch
    rng = np.random.default_rng(M + N + K)
    hA = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    hB = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    dA, dB = to_dev(hA), to_dev(hB)
    rows = np.sort(rng.choice(M, min(M, 48), replace=False))
    for prec, split in ((ls.PREC_FP32, 1), (ls.PREC_FP32, 0), (ls.PREC_BF16X6, 0)):
        dC = torch.full((M, N), float("nan"), device="cuda")
        ls.set_precision(prec)
        ls.set_splitk(split)
        ls.sgemm_mp(0, 0, dC, dA, dB, M, N, K)
        got = to_host(dC)[rows]
        if prec == ls.PREC_FP32 and split == 1:
            # no split-K: the GEMM_K = 320 blocked k-sequential order, bit for bit
            assert np.array_equal(got, orc.sgemm_kseq(hA[rows], hB, 0, kblock=320))
        else:
            assert normwise_err(got, orc.sgemm_f64(hA[rows], hB, 0)) <= 1e-6, (prec, split)
