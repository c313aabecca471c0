"""GPU parity of the plain FP32/FP64 paths, through the C ABI.

The plain kernels run one fused multiply-add chain per output element in
increasing k (the rounding order of the reference's KERNEL5x16 / KERNEL7x6
register tiles), so they are compared BIT-EXACTLY with the oracle's
k-sequential restatement, and additionally with the exact-math oracle under
the deterministic FP32 bound gamma_K (componentwise)."""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import componentwise_err, fp32_bound, normwise_err, to_dev, to_host

pytestmark = pytest.mark.gpu


def _run_sgemm(fn, transa, transb, A, B, M, N, K):
    import torch
    dA, dB = to_dev(A), to_dev(B)
    dC = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    fn(transa, transb, dC, dA, dB, M, N, K)
    return to_host(dC)


def test_config1_nt_80cubed_seed0():
    # LibShalom_sgemm(NoTrans, Trans), M=N=K=80, random_matrix() stream seed 0
    A, B = orc.gemm_inputs_f32(0, 80, 80, 80, 1)
    C = _run_sgemm(ls.sgemm, ls.NoTrans, ls.Trans, A, B, 80, 80, 80)
    assert np.array_equal(C, orc.sgemm_kseq(A, B, 1))
    ref = orc.sgemm_f64(A, B, 1)
    assert componentwise_err(C, ref, orc.sgemm_absprod(A, B, 1)) <= fp32_bound(80)
    # the reference's own (lane-split) order differs only by rounding
    r = orc.sgemm_nt_reforder(A, B)
    assert np.array_equal(C[5:], r[5:])
    assert normwise_err(C, r.astype(np.float64)) < 1e-6


TAILS = [(m, n, k) for m in (1, 2, 3, 5, 7, 8, 9, 16, 17)
         for n in (1, 4, 8, 13, 16, 17) for k in (1, 3, 8, 15, 17)]


@pytest.mark.parametrize("transb", [0, 1])
def test_sgemm_all_tails_bitexact(transb):
    for (M, N, K) in TAILS:
        A, B = orc.gemm_inputs_f32(M * 1000 + N * 10 + K, M, N, K, transb)
        C = _run_sgemm(ls.sgemm, 0, transb, A, B, M, N, K)
        assert np.array_equal(C, orc.sgemm_kseq(A, B, transb)), (M, N, K)


@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("n", list(range(8, 129, 8)))
def test_sgemm_cube_sweep(n, transb):
    # seeds 1..32: n/8 for NN, 16 + n/8 for NT
    seed = n // 8 + (16 if transb else 0)
    A, B = orc.gemm_inputs_f32(seed, n, n, n, transb)
    C = _run_sgemm(ls.sgemm, 0, transb, A, B, n, n, n)
    assert np.array_equal(C, orc.sgemm_kseq(A, B, transb))


@pytest.mark.parametrize("transa,transb", [(1, 0), (1, 1)])
def test_sgemm_transa(transa, transb):
    M, N, K = 37, 29, 41
    A = orc.uniform_f32(11, M * K).reshape(K, M)  # stored K x M
    B = orc.uniform_f32(12, K * N).reshape((N, K) if transb else (K, N))
    C = _run_sgemm(ls.sgemm, transa, transb, A, B, M, N, K)
    assert np.array_equal(C, orc.sgemm_kseq(A, B, transb, transa=1))


MP_SHAPES = [(64, 392, 576), (128, 98, 1152), (256, 49, 640), (512, 49, 960),
             (2048, 32, 2560), (32, 2048, 1024)]


@pytest.mark.parametrize("M,N,K", MP_SHAPES)
def test_sgemm_mp_bitexact_without_split(M, N, K):
    # no split-K: the GEMM_K = 320 fold reproduces the reference mp order
    A, B = orc.gemm_inputs_f32(M + N + K, M, N, K, 0)
    ls.set_splitk(1)
    try:
        C = _run_sgemm(ls.sgemm_mp, 0, 0, A, B, M, N, K)
    finally:
        ls.set_splitk(0)
    assert np.array_equal(C, orc.sgemm_kseq(A, B, 0, kblock=320))


@pytest.mark.parametrize("M,N,K", MP_SHAPES)
@pytest.mark.parametrize("transb", [0, 1])
def test_sgemm_mp_auto_split(M, N, K, transb):
    A, B = orc.gemm_inputs_f32(M * 3 + N + K, M, N, K, transb)
    C = _run_sgemm(ls.sgemm_mp, 0, transb, A, B, M, N, K)
    ref = orc.sgemm_f64(A, B, transb)
    assert componentwise_err(C, ref, orc.sgemm_absprod(A, B, transb)) <= fp32_bound(K)
    assert normwise_err(C, ref) <= 1e-6


def test_sgemm_mp_forced_split_and_ways():
    M, N, K = 96, 200, 3000
    A, B = orc.gemm_inputs_f32(77, M, N, K, 0)
    ref = orc.sgemm_f64(A, B, 0)
    ls.set_splitk(4)
    try:
        C = _run_sgemm(ls.sgemm_mp, 0, 0, A, B, M, N, K)
    finally:
        ls.set_splitk(0)
    assert normwise_err(C, ref) <= 1e-6
    # thread ways: a 2 x 3 partition of the tile grid, one-shot
    ls.set_splitk(1)
    try:
        ls.set_thread_ways(2, 3)
        C2 = _run_sgemm(ls.sgemm_mp, 0, 0, A, B, M, N, K)
    finally:
        ls.set_splitk(0)
    assert np.array_equal(C2, orc.sgemm_kseq(A, B, 0, kblock=320))


def test_thread_cap_does_not_change_results():
    M, N, K = 300, 260, 100
    A, B = orc.gemm_inputs_f32(5, M, N, K, 1)
    ls.set_thread_nums(3)
    try:
        C = _run_sgemm(ls.sgemm, 0, 1, A, B, M, N, K)
    finally:
        ls.set_thread_nums(0)
    assert np.array_equal(C, orc.sgemm_kseq(A, B, 1))


DGEMM_SIZES = [5, 9, 13, 16, 22, 23, 26, 32]


@pytest.mark.parametrize("transb", [0, 1])
def test_dgemm_config_sizes_bitexact(transb):
    import torch
    rng = np.random.default_rng(2)
    for M in DGEMM_SIZES:
        for N in (5, 16, 23, 32):
            for K in (5, 13, 32):
                A = rng.standard_normal((M, K)) * 10.0 ** rng.uniform(-3, 3)
                B = rng.standard_normal((N, K) if transb else (K, N)) * 10.0 ** rng.uniform(-3, 3)
                dC = torch.full((M, N), float("nan"), dtype=torch.float64, device="cuda")
                ls.dgemm(0, transb, dC, to_dev(A), to_dev(B), M, N, K)
                C = to_host(dC)
                assert np.array_equal(C, orc.dgemm_kseq(A, B, transb)), (M, N, K)
                assert normwise_err(C, orc.dgemm_ld(A, B, transb)) <= 1e-14


def test_dgemm_larger_and_tails():
    import torch
    rng = np.random.default_rng(3)
    for (M, N, K) in [(1, 1, 1), (7, 6, 4), (70, 130, 45), (257, 33, 19)]:
        A = rng.standard_normal((M, K))
        B = rng.standard_normal((K, N))
        dC = torch.empty((M, N), dtype=torch.float64, device="cuda")
        ls.dgemm(0, 0, dC, to_dev(A), to_dev(B), M, N, K)
        assert np.array_equal(to_host(dC), orc.dgemm_kseq(A, B, 0))


@pytest.mark.parametrize("transb", [0, 1])
@pytest.mark.parametrize("n", [8, 24, 40, 64, 96, 128])
def test_strided_batch_plain(n, transb):
    import torch
    count = 50
    A = orc.uniform_f32(n, count * n * n).reshape(count, n, n)
    B = orc.uniform_f32(n + 1, count * n * n).reshape(count, n, n)
    dC = torch.full((count, n, n), float("nan"), dtype=torch.float32, device="cuda")
    ls.sgemm_batched_strided(transb, n, n, n, 1.0, to_dev(A), n * n, to_dev(B), n * n, 0.0,
                             dC, n * n, count)
    C = to_host(dC)
    for g in range(0, count, 7):
        assert np.array_equal(C[g], orc.sgemm_kseq(A[g], B[g], transb)), g


def test_strided_batch_alpha_beta():
    import torch
    count, M, N, K = 20, 19, 23, 29
    A = orc.uniform_f32(1, count * M * K).reshape(count, M, K)
    B = orc.uniform_f32(2, count * K * N).reshape(count, K, N)
    C0 = orc.uniform_f32(3, count * M * N).reshape(count, M, N)
    dC = to_dev(C0)
    ls.sgemm_batched_strided(0, M, N, K, 0.5, to_dev(A), M * K, to_dev(B), K * N, 1.0, dC,
                             M * N, count)
    C = to_host(dC)
    for g in range(count):
        ref = orc.sgemm_f64(A[g], B[g], 0, alpha=0.5, beta=1.0, C=C0[g])
        assert normwise_err(C[g], ref) <= 1e-6


def _sgemm_entries(shapes, rng_seed=0, beta_choices=(0.0,)):
    """Builds a grouped batch in one device pool; returns host copies."""
    import torch
    sdt, _ = ls.entry_dtypes()
    rng = np.random.default_rng(rng_seed)
    As, Bs, C0s = [], [], []
    for i, (M, N, K, tb) in enumerate(shapes):
        As.append(orc.uniform_f32(2 * i + 1, M * K).reshape(M, K))
        Bs.append(orc.uniform_f32(2 * i + 2, K * N).reshape((N, K) if tb else (K, N)))
        C0s.append(orc.uniform_f32(10_000 + i, M * N).reshape(M, N))
    flatA = np.concatenate([a.ravel() for a in As])
    flatB = np.concatenate([b.ravel() for b in Bs])
    flatC = np.concatenate([c.ravel() for c in C0s])
    dA, dB, dC = to_dev(flatA), to_dev(flatB), to_dev(flatC)
    ent = np.zeros(len(shapes), sdt)
    oa = ob = oc = 0
    betas = []
    for i, (M, N, K, tb) in enumerate(shapes):
        beta = float(beta_choices[rng.integers(len(beta_choices))])
        betas.append(beta)
        ent[i] = (dA.data_ptr() + 4 * oa, dB.data_ptr() + 4 * ob, dC.data_ptr() + 4 * oc,
                  M, N, K, tb, 0, 0, 0, 1.0, beta, 0)
        oa += M * K
        ob += K * N
        oc += M * N
    dE = torch.from_numpy(ent.view(np.uint8)).cuda()
    return dict(As=As, Bs=Bs, C0s=C0s, betas=betas, dA=dA, dB=dB, dC=dC, dE=dE)


def _split(flat, shapes):
    out, o = [], 0
    for (M, N, K, tb) in shapes:
        out.append(flat[o:o + M * N].reshape(M, N))
        o += M * N
    return out


def test_grouped_batch_plain_mixed():
    rng = np.random.default_rng(5)
    shapes = []
    for _ in range(300):
        M, N, K = (int(np.exp(rng.uniform(np.log(4), np.log(256)))) for _ in range(3))
        shapes.append((M, N, K, int(rng.integers(2))))
    b = _sgemm_entries(shapes, beta_choices=(0.0, 1.0))
    ls.sgemm_batched(b["dE"], len(shapes))
    Cs = _split(to_host(b["dC"]), shapes)
    for i, (M, N, K, tb) in enumerate(shapes):
        if b["betas"][i] == 0.0:
            assert np.array_equal(Cs[i], orc.sgemm_kseq(b["As"][i], b["Bs"][i], tb)), i
        else:
            ref = orc.sgemm_f64(b["As"][i], b["Bs"][i], tb, beta=1.0, C=b["C0s"][i])
            assert normwise_err(Cs[i], ref) <= 1e-6, i


def _dgemm_runs(nruns, run, sizes, seed):
    """Batched DGEMM workload: runs of `run` products share one C block."""
    import torch
    _, ddt = ls.entry_dtypes()
    rng = np.random.default_rng(seed)
    As, Bs, Ms, Ns, Ks, offC = [], [], [], [], [], []
    C0 = []
    oc = 0
    for r in range(nruns):
        M, N = int(rng.choice(sizes)), int(rng.choice(sizes))
        C0.append(rng.standard_normal(M * N))
        for p in range(run):
            K = int(rng.choice(sizes))
            As.append(rng.standard_normal(M * K) * 10.0 ** rng.uniform(-3, 3))
            Bs.append(rng.standard_normal(K * N) * 10.0 ** rng.uniform(-3, 3))
            Ms.append(M); Ns.append(N); Ks.append(K); offC.append(oc)
        oc += M * N
    flatA, flatB, flatC = (np.concatenate(x) for x in (As, Bs, C0))
    dA, dB, dC = to_dev(flatA), to_dev(flatB), to_dev(flatC)
    ent = np.zeros(len(Ms), ddt)
    oa = ob = 0
    offA, offB = [], []
    for i in range(len(Ms)):
        ent[i] = (dA.data_ptr() + 8 * oa, dB.data_ptr() + 8 * ob, dC.data_ptr() + 8 * offC[i],
                  Ms[i], Ns[i], Ks[i], 0, 0, 0, 0, 0, 1.0, 1.0)
        offA.append(oa); offB.append(ob)
        oa += Ms[i] * Ks[i]
        ob += Ks[i] * Ns[i]
    dE = torch.from_numpy(ent.view(np.uint8)).cuda()
    i32 = lambda v: np.asarray(v, np.int32)
    i64 = lambda v: np.asarray(v, np.int64)
    ref = flatC.copy()
    orc.lib().orc_dgemm_batched_ld(len(Ms), i32(Ms), i32(Ns), i32(Ks), flatA, i64(offA), flatB,
                                   i64(offB), ref, i64(offC))
    blocks = sorted(set((offC[i], Ms[i] * Ns[i]) for i in range(len(Ms))))
    return dE, dC, ref, len(Ms), blocks


def run_errors(got, ref, blocks):
    """normwise error of every shared C block"""
    return [normwise_err(got[o:o + n], ref[o:o + n]) for (o, n) in blocks]


def test_dgemm_batched_runs_of_8():
    dE, dC, ref, count, blocks = _dgemm_runs(300, 8, [5, 9, 13, 16, 22, 23, 26, 32], 11)
    ls.dgemm_batched(dE, count)
    got = to_host(dC)
    assert max(run_errors(got, ref, blocks)) <= 1e-14


def test_invalid_precision_mode_on_gpu_does_not_launch():
    import torch
    dC = torch.zeros(4, 4, device="cuda")
    st = ls.sgemm(3, 0, dC, dC, dC, 4, 4, 4, check=False)
    assert st == ls.ERR_INVALID_VALUE
    assert torch.count_nonzero(dC).item() == 0
