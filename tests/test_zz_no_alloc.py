"""LibShalom_sgemm_mp_noalloc, through the C ABI.

The entry point is for callers that cannot allocate device memory (their GPU
memory belongs to another allocator, or a cudaMalloc in the middle of a call
is not acceptable).  It keeps the split-K partial sums in a fixed array
inside the library, so its results must match LibShalom_sgemm_mp run with
the same split factor (which keeps them in an allocated workspace).  This
file is collected last on purpose; it must pass alone in a fresh process and
after every other test."""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import normwise_err, to_dev, to_host

pytestmark = pytest.mark.gpu

SHAPES = [(64, 392, 1152, 4), (2048, 32, 2560, 8), (96, 200, 3000, 3), (33, 65, 700, 2)]


def _mp_reference(A, B, M, N, K, splits):
    import torch
    dC = torch.full((M, N), float("nan"), device="cuda")
    ls.set_splitk(splits)
    try:
        ls.sgemm_mp(0, 0, dC, to_dev(A), to_dev(B), M, N, K)
    finally:
        ls.set_splitk(0)
    return to_host(dC)


def test_noalloc_matches_sgemm_mp_two_calls_in_a_row():
    import torch
    for (M, N, K, splits) in SHAPES:
        for call in range(2):  # the second call reuses the array the first one left behind
            A, B = orc.gemm_inputs_f32(1000 * call + M + N + K, M, N, K, 0)
            dC = torch.full((M, N), float("nan"), device="cuda")
            ls.sgemm_mp_noalloc(0, 0, dC, to_dev(A), to_dev(B), M, N, K, splits)
            got = to_host(dC)
            want = _mp_reference(A, B, M, N, K, splits)
            assert not np.isnan(got).any()
            # same K slices, same kernels, same slice-ordered reduction
            assert np.array_equal(got, want), (M, N, K, splits, call)
            ref = orc.sgemm_f64(A, B, 0)
            assert normwise_err(got, ref) <= 1e-6


def test_noalloc_rejects_problems_beyond_the_array():
    import torch
    M, N, K = 1024, 1024, 64
    splits = ls.NOALLOC_SCRATCH_FLOATS // (M * N) + 1
    dC = torch.zeros((M, N), device="cuda")
    dA = torch.ones((M, K), device="cuda")
    dB = torch.ones((K, N), device="cuda")
    st = ls.sgemm_mp_noalloc(0, 0, dC, dA, dB, M, N, K, splits, check=False)
    assert st == ls.ERR_INVALID_VALUE
    torch.cuda.synchronize()
    assert torch.count_nonzero(dC).item() == 0  # nothing was launched


def test_noalloc_empty_and_short_k():
    """K = 0 writes C = 0 (an empty sum) instead of dividing by a zero K slice
    on the host; K below the split factor runs as one slice."""
    import torch
    for (M, N, K, splits) in [(7, 9, 0, 3), (12, 5, 3, 8), (40, 24, 1, 2)]:
        dC = torch.full((M, N), float("nan"), device="cuda")
        A, B = orc.gemm_inputs_f32(M * N + K, M, N, max(K, 1), 0)
        A, B = A[:, :K].copy(), B[:K, :].copy()
        ls.sgemm_mp_noalloc(0, 0, dC, to_dev(A) if K else None, to_dev(B) if K else None,
                            M, N, K, splits)
        got = to_host(dC)
        if K == 0:
            assert np.array_equal(got, np.zeros((M, N), np.float32))
        else:
            assert np.array_equal(got, _mp_reference(A, B, M, N, K, splits)), (M, N, K)
