"""GPU parity of deferred drop-in calls (LibShalom_defer_begin / _flush: the
calls are recorded in a host-pinned ring and run as grouped batches), through
the C ABI.

Plain FP32 and FP64 FMA results are compared BIT-EXACTLY with the direct
calls (one fused multiply-add chain per element in increasing k on both
paths); split-BF16 x6 within normwise max|C - C64| / max|C64| <= 1e-6 against
the FP64 oracle."""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import normwise_err, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture
def reset():
    yield
    if ls.defer_pending():
        ls.defer_flush(check=False)
    ls.set_precision(ls.PREC_FP32)
    ls.set_dgemm_method(ls.DGEMM_FMA, 0)
    ls.set_sync(True)
    ls.set_stream(None)


def _problems(rng, count):
    out = []
    for i in range(count):
        M, N, K = (int(v) for v in rng.integers(1, 97, size=3))
        tb = int(rng.integers(2))
        dbl = i % 4 == 3
        dt = np.float64 if dbl else np.float32
        A = rng.uniform(-1, 1, size=(M, K)).astype(dt)
        B = rng.uniform(-1, 1, size=(N, K) if tb else (K, N)).astype(dt)
        out.append((dbl, tb, M, N, K, A, B))
    return out


def test_deferred_calls_match_direct_calls(reset):
    import torch
    rng = np.random.default_rng(31)
    probs = _problems(rng, 240)
    dev = [(to_dev(A), to_dev(B)) for (_, _, _, _, _, A, B) in probs]
    outs = [torch.full((M, N), float("nan"), device="cuda",
                       dtype=torch.float64 if dbl else torch.float32)
            for (dbl, _, M, N, _, _, _) in probs]
    ls.defer_begin()
    for (dbl, tb, M, N, K, _, _), (dA, dB), C in zip(probs, dev, outs):
        (ls.dgemm if dbl else ls.sgemm)(0, tb, C, dA, dB, M, N, K)
    assert ls.defer_pending() == len(probs)  # independent calls: nothing flushed early
    ls.defer_flush()
    assert ls.defer_pending() == 0
    for i, ((dbl, tb, M, N, K, A, B), (dA, dB), C) in enumerate(zip(probs, dev, outs)):
        direct = torch.empty_like(C)
        (ls.dgemm if dbl else ls.sgemm)(0, tb, direct, dA, dB, M, N, K)
        assert torch.equal(C, direct), i
        if i % 16 == 0:
            ref = (orc.dgemm_kseq if dbl else orc.sgemm_kseq)(A, B, tb)
            assert np.array_equal(to_host(C), ref), i


def test_deferred_hazards_keep_call_order(reset):
    import torch
    rng = np.random.default_rng(7)
    n = 24
    mat = lambda: to_dev(rng.uniform(-1, 1, size=(n, n)).astype(np.float32))  # noqa: E731
    X, Y, Z = mat(), mat(), mat()
    Y0 = Y.clone()
    C1, C2, C3 = (torch.empty(n, n, device="cuda") for _ in range(3))
    ls.defer_begin()
    ls.sgemm(0, 0, C1, X, Y, n, n, n)   # a: C1 = X Y
    ls.sgemm(0, 0, C2, C1, Y, n, n, n)  # b: reads C1, which a writes: a is launched first
    assert ls.defer_pending() == 1
    ls.sgemm(0, 0, Y, X, X, n, n, n)    # c: writes Y, which b reads: b is launched first
    assert ls.defer_pending() == 1
    ls.sgemm(0, 0, C3, X, X, n, n, n)   # d: independent
    assert ls.defer_pending() == 2
    ls.sgemm(0, 0, Y, X, Z, n, n, n)    # e: writes Y again, not right after c: flush
    assert ls.defer_pending() == 1
    ls.sgemm(0, 0, Y, Z, Z, n, n, n)    # f: same C right after e: applied in order
    assert ls.defer_pending() == 2
    ls.defer_flush()
    tol = dict(rtol=1e-5, atol=1e-4)
    c1 = X @ Y0
    assert torch.allclose(C1, c1, **tol)
    assert torch.allclose(C2, c1 @ Y0, **tol)
    assert torch.allclose(C3, X @ X, **tol)
    assert torch.allclose(Y, Z @ Z, **tol)


def test_deferred_transa_call_runs_directly_in_order(reset):
    import torch
    A, B = orc.gemm_inputs_f32(5, 40, 30, 20, 0)
    At = np.ascontiguousarray(A.T)  # K x M storage for transa
    dA, dAt, dB = to_dev(A), to_dev(At), to_dev(B)
    C1 = torch.empty(40, 30, device="cuda")
    C2 = torch.empty(40, 30, device="cuda")
    ls.defer_begin()
    ls.sgemm(0, 0, C1, dA, dB, 40, 30, 20)
    ls.sgemm(1, 0, C2, dAt, dB, 40, 30, 20)  # cannot be recorded: flush, then run
    assert ls.defer_pending() == 0
    ls.defer_flush()
    ref = orc.sgemm_kseq(A, B, 0)
    assert np.array_equal(to_host(C1), ref)
    assert np.array_equal(to_host(C2), orc.sgemm_kseq(At, B, 0, transa=1))


def test_deferred_large_call_runs_directly(reset):
    """A call above 128^3 (M N K) is not recorded: the pending calls are
    launched, then it runs on the direct path."""
    import torch
    A, B = orc.gemm_inputs_f32(8, 16, 16, 16, 0)
    dA, dB = to_dev(A), to_dev(B)
    C1 = torch.empty(16, 16, device="cuda")
    M, N, K = 300, 200, 100
    L, R = orc.gemm_inputs_f32(9, M, N, K, 0)
    dL, dR = to_dev(L), to_dev(R)
    C2 = torch.empty(M, N, device="cuda")
    ls.defer_begin()
    ls.sgemm(0, 0, C1, dA, dB, 16, 16, 16)
    assert ls.defer_pending() == 1
    ls.sgemm(0, 0, C2, dL, dR, M, N, K)
    assert ls.defer_pending() == 0
    ls.defer_flush()
    assert np.array_equal(to_host(C1), orc.sgemm_kseq(A, B, 0))
    assert np.array_equal(to_host(C2), orc.sgemm_kseq(L, R, 0))


def test_deferred_split_bf16_on_a_side_stream(reset):
    import torch
    rng = np.random.default_rng(11)
    s = torch.cuda.Stream()
    ls.set_stream(s)
    ls.set_sync(False)
    ls.set_precision(ls.PREC_BF16X6)
    probs = [p for p in _problems(rng, 60) if not p[0]]
    outs, keep = [], []  # operands stay allocated until the flush has run
    ls.defer_begin()
    with torch.cuda.stream(s):
        for (_, tb, M, N, K, A, B) in probs:
            C = torch.full((M, N), float("nan"), device="cuda")
            dA, dB = to_dev(A), to_dev(B)
            ls.sgemm_mp(0, tb, C, dA, dB, M, N, K)
            outs.append(C)
            keep += [dA, dB]
    ls.defer_flush()
    ls.synchronize()
    for (_, tb, M, N, K, A, B), C in zip(probs, outs):
        assert normwise_err(to_host(C), orc.sgemm_f64(A, B, tb)) <= 1e-6


def _entries(sdt, rows):
    """Device buffer of SgemmEntry records: rows of (A, B, C, M, N, K, transb)."""
    ent = np.array([(a.data_ptr(), b.data_ptr(), c.data_ptr(), M, N, K, tb, 0, 0, 0, 1.0, 0.0, 0)
                    for (a, b, c, M, N, K, tb) in rows], sdt)
    return to_dev(ent.view(np.uint8))


def test_batched_and_ex_calls_run_after_pending_calls(reset):
    """Calls that are not recorded (a grouped batch, an _ex call) read a C that
    a pending recorded call writes: they must launch the pending calls first."""
    import torch
    n = 20
    A, B = orc.gemm_inputs_f32(21, n, n, n, 0)
    D = orc.uniform_f32(22, n * n).reshape(n, n)
    dA, dB, dD = to_dev(A), to_dev(B), to_dev(D)
    X = torch.full((n, n), float("nan"), device="cuda")
    Y = torch.full((n, n), float("nan"), device="cuda")
    Z = torch.full((n, n), float("nan"), device="cuda")
    sdt, _ = ls.entry_dtypes()
    ent = _entries(sdt, [(X, dD, Y, n, n, n, 0)])  # Y = X D
    ls.defer_begin()
    ls.sgemm(0, 0, X, dA, dB, n, n, n)  # recorded: X = A B
    assert ls.defer_pending() == 1
    ls.sgemm_batched(ent, 1)            # reads X: the recorded call runs first
    assert ls.defer_pending() == 0
    ls.sgemm(0, 0, X, dA, dB, n, n, n)  # recorded again
    ls.sgemm_ex(0, 0, n, n, n, 1.0, X, n, dD, n, 0.0, Z, n)  # Z = X D, after the pending call
    assert ls.defer_pending() == 0
    ls.defer_flush()
    x = orc.sgemm_kseq(A, B, 0)
    assert np.array_equal(to_host(X), x)
    assert normwise_err(to_host(Y), orc.sgemm_f64(x, D, 0)) <= 1e-6
    assert normwise_err(to_host(Z), orc.sgemm_f64(x, D, 0)) <= 1e-6


def test_setters_and_finalize_launch_pending_calls(reset):
    """Changing the precision launches the pending calls under the precision
    they were recorded with; finalize runs what is still pending."""
    import torch
    A, B = orc.gemm_inputs_f32(23, 33, 17, 29, 0)
    dA, dB = to_dev(A), to_dev(B)
    C1 = torch.full((33, 17), float("nan"), device="cuda")
    C2 = torch.full((33, 17), float("nan"), device="cuda")
    ls.defer_begin()
    ls.sgemm_mp(0, 0, C1, dA, dB, 33, 17, 29)   # recorded under plain FP32
    ls.set_precision(ls.PREC_BF16X6)           # launches it first
    assert ls.defer_pending() == 0
    ls.set_precision(ls.PREC_FP32)
    ls.sgemm(0, 0, C2, dA, dB, 33, 17, 29)
    assert ls.defer_pending() == 1
    ls.finalize()                              # runs the pending call, then frees
    assert ls.last_error() == ls.SUCCESS
    assert ls.defer_pending() == 0
    torch.cuda.synchronize()
    ref = orc.sgemm_kseq(A, B, 0)
    assert np.array_equal(to_host(C1), ref)  # plain FP32 result, bit for bit
    assert np.array_equal(to_host(C2), ref)
