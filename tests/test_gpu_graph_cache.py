"""Graph cache of repeated single / mp calls (LibShalom_set_graph_cache):
replays give the same results as direct calls while the data behind the
pointers changes, across precision modes and a workspace that grows.

Tolerance: plain FP32 bit-exact with the k-sequential restatement; split-BF16
x6 normwise <= 1e-6; FP64 bit-exact with the k-sequential FMA restatement."""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import normwise_err, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture
def cached():
    import torch
    s = torch.cuda.Stream()
    ls.set_stream(s)
    ls.set_graph_cache(True)
    yield s
    ls.set_graph_cache(False)
    ls.set_precision(ls.PREC_FP32)
    ls.set_stream(None)


@pytest.mark.parametrize("sync", [True, False])
def test_single_call_replays(cached, sync):
    import torch
    M = N = K = 80
    dA = torch.empty((M, K), device="cuda")
    dB = torch.empty((N, K), device="cuda")
    dC = torch.empty((M, N), device="cuda")
    ls.set_sync(sync)
    try:
        for it in range(5):  # run, capture, then three replays
            A = orc.uniform_f32(40 + it, M * K).reshape(M, K)
            B = orc.uniform_f32(60 + it, N * K).reshape(N, K)
            with torch.cuda.stream(cached):
                dA.copy_(torch.from_numpy(A))
                dB.copy_(torch.from_numpy(B))
            ls.sgemm(0, 1, dC, dA, dB, M, N, K)
            cached.synchronize()
            assert np.array_equal(to_host(dC), orc.sgemm_kseq(A, B, 1)), it
    finally:
        ls.set_sync(True)


def test_mp_tensor_core_and_workspace_growth(cached):
    import torch
    M, N, K = 512, 49, 4608
    dA = torch.empty((M, K), device="cuda")
    dB = torch.empty((K, N), device="cuda")
    dC = torch.empty((M, N), device="cuda")
    ls.set_precision(ls.PREC_BF16X6)
    for it in range(4):
        if it == 2:
            # a larger split-K call grows the workspace: the cached graph of
            # the first shape must be recaptured, not replayed
            big = torch.empty((20480, 32), device="cuda")
            bA = torch.rand((20480, 20480), device="cuda")
            bB = torch.rand((20480, 32), device="cuda")
            ls.sgemm_mp(0, 0, big, bA, bB, 20480, 32, 20480)
            del bA, bB, big
        A, B = orc.gemm_inputs_f32(70 + it, M, N, K, 0)
        with torch.cuda.stream(cached):
            dA.copy_(torch.from_numpy(A))
            dB.copy_(torch.from_numpy(B))
        ls.sgemm_mp(0, 0, dC, dA, dB, M, N, K)
        cached.synchronize()
        assert normwise_err(to_host(dC), orc.sgemm_f64(A, B, 0)) <= 1e-6, it


def test_dgemm_replays(cached):
    import torch
    M, N, K = 23, 26, 32
    dA = torch.empty((M, K), device="cuda", dtype=torch.float64)
    dB = torch.empty((K, N), device="cuda", dtype=torch.float64)
    dC = torch.empty((M, N), device="cuda", dtype=torch.float64)
    rng = np.random.default_rng(3)
    for it in range(4):
        A = rng.standard_normal((M, K))
        B = rng.standard_normal((K, N))
        with torch.cuda.stream(cached):
            dA.copy_(torch.from_numpy(A))
            dB.copy_(torch.from_numpy(B))
        ls.dgemm(0, 0, dC, dA, dB, M, N, K)
        cached.synchronize()
        assert normwise_err(to_host(dC), orc.dgemm_ld(A, B, 0)) <= 1e-15, it
