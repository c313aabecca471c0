"""Failure detection on the GPU without a fault: the tensor-core kernels'
bounded mbarrier waits give up, report through a device status word and let
the kernel return.  LibShalom_selftest_wait_expiry makes one such wait run out
(an mbarrier nothing arrives at) and the call must return
LIBSHALOM_ERR_DEVICE_TIMEOUT; the context stays usable afterwards."""
import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("iterations", [0, 100, 20000])
def test_expired_wait_is_reported_and_context_survives(iterations):
    import torch
    assert ls.selftest_wait_expiry(iterations) == ls.ERR_DEVICE_TIMEOUT
    assert ls.last_error() == ls.ERR_DEVICE_TIMEOUT
    # the status word was cleared and the GPU still computes
    A, B = orc.gemm_inputs_f32(3, 40, 24, 56, 0)
    dC = torch.full((40, 24), float("nan"), device="cuda")
    ls.set_precision(ls.PREC_BF16X6)
    try:
        ls.sgemm_mp(0, 0, dC, to_dev(A), to_dev(B), 40, 24, 56)
    finally:
        ls.set_precision(ls.PREC_FP32)
    ref = orc.sgemm_f64(A, B, 0)
    assert np.max(np.abs(to_host(dC) - ref)) / np.max(np.abs(ref)) <= 1e-6


def test_negative_limit_rejected():
    assert ls.selftest_wait_expiry(-1) == ls.ERR_INVALID_VALUE
