"""GPU parity of the front ends: plain calls with explicit leading dimensions
and alpha / beta, the DBCSR-style DGEMM stack, and the convolution (implicit
GEMM in FP32, im2col + mp GEMM in the split-BF16 modes).

Tolerances (normwise max|C - C_ref| / max|C_ref|): FP32 plain and split-BF16
x6 <= 1e-6, FP64 <= 1e-14, against the FP64 / long-double oracle (torch FP64
on the host for the convolution)."""
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
    ls.set_dgemm_method(ls.DGEMM_FMA, 0)


def _padded(rng, rows, cols, ld, dtype):
    buf = (rng.uniform(-1, 1, size=(rows, ld))).astype(dtype)
    return buf, buf[:, :cols]


@pytest.mark.parametrize("transa,transb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(37, 53, 71), (128, 20, 700), (5, 300, 33)])
def test_sgemm_ex(transa, transb, M, N, K, reset):
    rng = np.random.default_rng(M + 3 * N + 7 * K + transa + 2 * transb)
    Ab, A = _padded(rng, K if transa else M, M if transa else K, (M if transa else K) + 3,
                    np.float32)
    Bb, B = _padded(rng, N if transb else K, K if transb else N, (K if transb else N) + 5,
                    np.float32)
    Cb, C0 = _padded(rng, M, N, N + 2, np.float32)
    ref = orc.sgemm_f64(np.ascontiguousarray(A), np.ascontiguousarray(B), transb, alpha=-0.75,
                        beta=1.5, C=np.ascontiguousarray(C0), transa=transa)
    dC = to_dev(Cb)
    ls.sgemm_ex(transa, transb, M, N, K, -0.75, to_dev(Ab), Ab.shape[1], to_dev(Bb),
                Bb.shape[1], 1.5, dC, Cb.shape[1])
    got = to_host(dC)
    assert normwise_err(got[:, :N], ref) <= 1e-6
    assert np.array_equal(got[:, N:], Cb[:, N:])  # padding untouched
    if not transa:
        ls.set_precision(ls.PREC_BF16X6)
        dC = to_dev(Cb)
        ls.sgemm_ex(transa, transb, M, N, K, -0.75, to_dev(Ab), Ab.shape[1], to_dev(Bb),
                    Bb.shape[1], 1.5, dC, Cb.shape[1])
        assert normwise_err(to_host(dC)[:, :N], ref) <= 1e-6


@pytest.mark.parametrize("transa,transb", [(0, 0), (1, 1)])
def test_dgemm_ex(transa, transb, reset):
    M, N, K = 45, 61, 90
    rng = np.random.default_rng(17)
    Ab, A = _padded(rng, K if transa else M, M if transa else K, (M if transa else K) + 1,
                    np.float64)
    Bb, B = _padded(rng, N if transb else K, K if transb else N, (K if transb else N) + 3,
                    np.float64)
    Cb, C0 = _padded(rng, M, N, N + 1, np.float64)
    ref = orc.dgemm_ld(np.ascontiguousarray(A), np.ascontiguousarray(B), transb, alpha=2.0,
                       beta=-1.0, C=np.ascontiguousarray(C0), transa=transa)
    dC = to_dev(Cb)
    ls.dgemm_ex(transa, transb, M, N, K, 2.0, to_dev(Ab), Ab.shape[1], to_dev(Bb), Bb.shape[1],
                -1.0, dC, Cb.shape[1])
    assert normwise_err(to_host(dC)[:, :N], ref) <= 1e-14


def test_ex_rejects_short_leading_dimension():
    import torch
    d = torch.zeros(64, device="cuda")
    st = ls.sgemm_ex(0, 0, 4, 4, 4, 1.0, d, 3, d, 4, 0.0, d, 4, check=False)
    assert st == ls.ERR_INVALID_VALUE


@pytest.mark.parametrize("method", [ls.DGEMM_FMA, ls.DGEMM_DMMA])
@pytest.mark.parametrize("uniform", [True, False])
def test_dgemm_stack(method, uniform, reset):
    """pools + offsets; consecutive products with one C offset accumulate"""
    import torch
    rng = np.random.default_rng(23 + uniform)
    sizes = [5, 13, 23, 32]
    nruns, run = 120, 4
    Ms, Ns, Ks, ao, bo, co = [], [], [], [], [], []
    a_pool, b_pool, c_blocks = [], [], []
    oa = ob = oc = 0
    for r in range(nruns):
        M = 13 if uniform else int(rng.choice(sizes))
        N = 23 if uniform else int(rng.choice(sizes))
        c_blocks.append(rng.standard_normal(M * N))
        for p in range(run):
            K = 9 if uniform else int(rng.choice(sizes))
            a_pool.append(rng.standard_normal(M * K))
            b_pool.append(rng.standard_normal(K * N))
            Ms.append(M); Ns.append(N); Ks.append(K)
            ao.append(oa); bo.append(ob); co.append(oc)
            oa += M * K
            ob += K * N
        oc += M * N
    A, B, C0 = (np.concatenate(x) for x in (a_pool, b_pool, c_blocks))
    dC = to_dev(C0)
    i64 = lambda v: to_dev(np.asarray(v, np.int64))  # noqa: E731
    i32 = lambda v: to_dev(np.asarray(v, np.int32))  # noqa: E731
    ls.set_dgemm_method(method, 0)
    if uniform:
        ls.dgemm_stack(to_dev(A), to_dev(B), dC, i64(ao), i64(bo), i64(co), len(Ms),
                       m=13, n=23, k=9, alpha=1.0, beta=1.0)
    else:
        ls.dgemm_stack(to_dev(A), to_dev(B), dC, i64(ao), i64(bo), i64(co), len(Ms),
                       M=i32(Ms), N=i32(Ns), K=i32(Ks), alpha=1.0, beta=1.0)
    torch.cuda.synchronize()
    got = to_host(dC)
    ref = C0.copy()
    for i in range(len(Ms)):
        M, N, K = Ms[i], Ns[i], Ks[i]
        c = ref[co[i]:co[i] + M * N].reshape(M, N)
        c[:] = orc.dgemm_ld(A[ao[i]:ao[i] + M * K].reshape(M, K),
                            B[bo[i]:bo[i] + K * N].reshape(K, N), 0, beta=1.0, C=c.copy())
    for r in range(nruns):
        i = r * run
        M, N = Ms[i], Ns[i]
        o = co[i]
        assert normwise_err(got[o:o + M * N], ref[o:o + M * N]) <= 1e-14, r


@pytest.mark.parametrize("n,c,h,w,oc,kh,kw,sh,sw,ph,pw", [
    (3, 5, 11, 23, 7, 3, 5, 2, 1, 0, 2),     # rectangular kernel, mixed stride / padding
    (2, 64, 30, 30, 96, 3, 3, 1, 1, 1, 1),   # K = 576: 36 K-slabs, 2 x 15 output tiles
    (1, 1, 9, 9, 1, 9, 9, 1, 1, 4, 4),       # one channel, kernel as large as the image
    (4, 8, 13, 13, 130, 1, 1, 3, 3, 0, 0),   # 1 x 1, stride 3, oc past one 64-row tile
    (2, 256, 14, 14, 64, 3, 3, 1, 1, 1, 1),  # K = 2304: the GEMM_K = 320 blocked chains
])
def test_sconv2d_implicit_fp32(n, c, h, w, oc, kh, kw, sh, sw, ph, pw, reset):
    """FP32 convolution as an implicit GEMM (the tile loader gathers the im2col
    columns from the image; no column buffer), against torch FP64 conv2d."""
    import torch
    rng = np.random.default_rng(n + c + h + w + oc)
    x = rng.uniform(-1, 1, size=(n, c, h, w)).astype(np.float32)
    wt = rng.uniform(-1, 1, size=(oc, c, kh, kw)).astype(np.float32)
    ref = torch.nn.functional.conv2d(torch.from_numpy(x).double(), torch.from_numpy(wt).double(),
                                     stride=(sh, sw), padding=(ph, pw)).numpy()
    y = torch.full(ref.shape, float("nan"), device="cuda", dtype=torch.float32)
    ls.set_precision(ls.PREC_FP32)
    ls.sconv2d_nchw(to_dev(x), n, c, h, w, to_dev(wt), oc, kh, kw, sh, sw, ph, pw, y)
    assert normwise_err(to_host(y), ref) <= 1e-6


@pytest.mark.parametrize("prec", [ls.PREC_FP32, ls.PREC_BF16X6])
@pytest.mark.parametrize("n,c,h,w,oc,k,s,p", [(2, 3, 17, 19, 8, 3, 1, 1), (1, 16, 14, 14, 32, 1, 1, 0),
                                              (2, 4, 20, 20, 6, 5, 2, 2), (1, 64, 8, 8, 64, 3, 2, 1)])
def test_sconv2d_nchw(prec, n, c, h, w, oc, k, s, p, reset):
    import torch
    rng = np.random.default_rng(n + c + h + oc + k)
    x = rng.uniform(-1, 1, size=(n, c, h, w)).astype(np.float32)
    wt = rng.uniform(-1, 1, size=(oc, c, k, k)).astype(np.float32)
    ref = torch.nn.functional.conv2d(torch.from_numpy(x).double(), torch.from_numpy(wt).double(),
                                     stride=s, padding=p).numpy()
    y = torch.full(ref.shape, float("nan"), device="cuda", dtype=torch.float32)
    ls.set_precision(prec)
    ls.sconv2d_nchw(to_dev(x), n, c, h, w, to_dev(wt), oc, k, k, s, s, p, p, y)
    assert normwise_err(to_host(y), ref) <= 1e-6
