"""GPU plain kernels against the golden fixtures: the outputs of the
reference's own instructions (tests/golden/make_golden.py executes them on
oracle/neon_emu.py), through the C ABI.

SGEMM NN (SGEMM_NN_L1 / SGEMM_NN): bit-exact.  LibShalom_sgemm_mp (the
reference's NGM driver with its GEMM_K = 320 blocks, SMM_NN_new.c:92-280):
bit-exact outside the reference's defective 12-column edge.  SGEMM NT (SGEMM_NT, incl. the
80^3 seed-0 call LibShalom_sgemm(NoTrans, Trans)): bit-exact on every row the
reference computes k-sequentially (rows >= 5 of each strip), and within the
FP32 bound elsewhere (its first row block uses a lane-split order).  DGEMM
(DGEMM_NN): bit-exact on every column the reference computes k-sequentially,
within 1e-14 normwise on its lane-split N1 column; elements the reference
leaves unwritten or gets wrong are compared with the exact math instead."""
import os

import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import componentwise_err, fp32_bound, normwise_err, to_dev, to_host
from tests.test_oracle import FIXTURES, load_fixture

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_gpu_matches_reference_fixture(path):
    import torch
    kind, A, B, Cref = load_fixture(path)
    M, N = Cref.shape
    K = A.shape[1]
    if kind == "sgemm_mp_ngm_ref":
        # LibShalom_sgemm_mp without split-K: the GEMM_K = 320 blocked order of
        # the reference's NGM driver, bit for bit outside its defective edge
        dC = torch.full((M, N), float("nan"), device="cuda")
        ls.set_splitk(1)
        try:
            ls.sgemm_mp(ls.NoTrans, ls.NoTrans, dC, to_dev(A), to_dev(B), M, N, K)
        finally:
            ls.set_splitk(0)
        C = to_host(dC)
        ok = np.ones(N, bool)
        ok[np.load(path)["edge_cols"]] = False
        assert np.array_equal(C[:, ok], Cref[:, ok])
        ref = orc.sgemm_f64(A, B, 0)
        assert componentwise_err(C, ref, orc.sgemm_absprod(A, B, 0)) <= fp32_bound(K)
        return
    if kind.startswith("sgemm"):
        tb = 1 if kind == "sgemm_nt_ref" else 0
        dC = torch.full((M, N), float("nan"), device="cuda")
        ls.sgemm(ls.NoTrans, tb, dC, to_dev(A), to_dev(B), M, N, K)
        C = to_host(dC)
        if tb == 0:
            assert np.array_equal(C, Cref)
        else:
            rows = np.arange(M) >= 5  # N % 16 == 0 here: rows 0..4 are the lane-split block
            assert np.array_equal(C[rows], Cref[rows])
            ref = orc.sgemm_f64(A, B, 1)
            assert componentwise_err(C, ref, orc.sgemm_absprod(A, B, 1)) <= fp32_bound(K)
            assert normwise_err(C, Cref.astype(np.float64)) <= 1e-6
    else:
        dC = torch.full((M, N), float("nan"), dtype=torch.float64, device="cuda")
        ls.dgemm(ls.NoTrans, ls.NoTrans, dC, to_dev(A), to_dev(B), M, N, K)
        C = to_host(dC)
        exact = orc.dgemm_ld(A, B, 0)
        correct = ~np.isnan(Cref) & (np.abs(Cref - exact) <= 1e-12 * np.abs(exact).max())
        kseq_cols = np.ones(N, bool)
        if N % 2 == 1:
            kseq_cols[N - 1] = False  # the reference's lane-split N1 column
        mask = correct & kseq_cols[None, :]
        assert np.array_equal(C[mask], Cref[mask])
        assert normwise_err(C, exact) <= 1e-14
