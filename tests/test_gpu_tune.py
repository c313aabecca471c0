"""The measured shape-class table (libshalom_b200/autotune.py ->
csrc/ls_tune_table.inc) is what the single / mp schedulers use, and the
schedules it picks give the same accuracy as the cost model's.

Tolerance: normwise max|C - C64| / max|C64| <= 1e-6 against the FP64 oracle
(plain FP32 and split-BF16 x6)."""
import os
import re

import numpy as np
import pytest

import libshalom_b200 as ls
from libshalom_b200.autotune import KIND, half_octave
from oracle import oracle as orc
from tests._util import normwise_err, to_dev, to_host

pytestmark = pytest.mark.gpu

TABLE = os.path.join(os.path.dirname(ls.__file__), "csrc", "ls_tune_table.inc")


def _table():
    rows = {}
    for line in open(TABLE):
        m = re.match(r"\{(\d+), (\d+), (\d+), (\d+), (-?\d+), (\d+)\}", line.strip())
        if m:
            k, mb, nb, kb, cfg, sp = (int(v) for v in m.groups())
            rows[(k, mb, nb, kb)] = (cfg, sp)
    return rows


@pytest.fixture
def reset():
    yield
    ls.set_autotune(True)
    ls.set_tile_config(-1)
    ls.set_splitk(0)
    ls.set_precision(ls.PREC_FP32)


def test_library_holds_the_table(reset):
    rows = _table()
    assert rows, "empty tuning table"
    assert ls.get_plan()[2] == len(rows)


@pytest.mark.parametrize("kind,prec", [("s_mp", ls.PREC_FP32), ("tc_bf16x6", ls.PREC_BF16X6)])
@pytest.mark.parametrize("M,N,K", [(512, 49, 4608), (256, 196, 2304), (64, 3136, 576)])
def test_table_schedule_used_and_accurate(kind, prec, M, N, K, reset):
    import torch
    rows = _table()
    key = (KIND[kind], half_octave(M), half_octave(N), half_octave(K))
    if key not in rows:
        pytest.skip("shape class not in the table")
    cfg, sp = rows[key]
    A, B = orc.gemm_inputs_f32(M + N + K, M, N, K, 0)
    ref = orc.sgemm_f64(A, B, 0)
    dA, dB = to_dev(A), to_dev(B)
    ls.set_precision(prec)
    outs = []
    for tuned in (True, False):
        ls.set_autotune(tuned)
        dC = torch.full((M, N), float("nan"), device="cuda")
        ls.sgemm_mp(0, 0, dC, dA, dB, M, N, K)
        plan = ls.get_plan()[:2]
        if tuned:
            assert plan[0] == cfg and plan[1] == sp, (plan, (cfg, sp))
        err = normwise_err(to_host(dC), ref)
        assert err <= 1e-6, (tuned, plan, err)
        outs.append(plan)


def test_forced_tile_config(reset):
    import torch
    M = N = K = 96
    A, B = orc.gemm_inputs_f32(3, M, N, K, 0)
    dA, dB = to_dev(A), to_dev(B)
    dC = torch.zeros((M, N), device="cuda")
    ref = orc.sgemm_kseq(A, B, 0)
    for cfg in range(7):
        ls.set_tile_config(cfg)
        ls.sgemm(0, 0, dC, dA, dB, M, N, K)
        assert ls.get_plan()[0] == cfg
        # every tile shape keeps the reference's per-element FMA order
        assert np.array_equal(to_host(dC), ref), cfg
    # FP64 has four tile shapes: a fifth is an error, not a silent fallback
    ls.set_tile_config(5)
    dD = torch.zeros((M, N), device="cuda", dtype=torch.float64)
    st = ls.dgemm(0, 0, dD, to_dev(A.astype(np.float64)), to_dev(B.astype(np.float64)), M, N, K,
                  check=False)
    assert st == ls.ERR_INVALID_VALUE
    assert ls.lib().LibShalom_set_tile_config(7) == ls.ERR_INVALID_VALUE
