"""CPU checks of the C-ABI boundary: the library loads, exports exactly what
include/LibShalom.h declares, the entry-structure layout matches the header,
and argument validation answers before any device work."""
import ctypes
import os
import re
import subprocess

import pytest

import libshalom_b200 as ls

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "LibShalom.h")


def _declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"LIBSHALOM_API\s+[^;(]*?\b(LibShalom_\w+)\s*\(", src)))


def _exported():
    out = subprocess.run(["nm", "-D", "--defined-only", ls.LIB_PATH], check=True,
                         capture_output=True, text=True).stdout
    return sorted(set(m.group(1) for m in re.finditer(r" T (LibShalom_\w+)", out)))


def test_library_loads():
    assert os.path.exists(ls.LIB_PATH)
    ls.lib()


def test_exports_match_header():
    declared = _declared()
    assert declared, "no declarations parsed"
    assert declared == _exported()
    assert sorted(ls.EXPORTED) == declared


def test_reference_entry_points_present():
    # NN_LIB/LibShalom.h:22,27,38,40,41
    for name in ("LibShalom_sgemm", "LibShalom_sgemm_mp", "LibShalom_dgemm",
                 "LibShalom_set_thread_nums", "LibShalom_set_thread_ways"):
        assert name in _exported()


def test_entry_layout_matches_header(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "LibShalom.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\","
        "sizeof(LibShalom_sgemm_entry), sizeof(LibShalom_dgemm_entry),"
        "offsetof(LibShalom_sgemm_entry, M), offsetof(LibShalom_sgemm_entry, alpha),"
        "offsetof(LibShalom_dgemm_entry, alpha), offsetof(LibShalom_dgemm_entry, ldc));"
        "return 0;}\n")
    exe = tmp_path / "sz"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(prog), "-o",
                    str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True,
                                           text=True).stdout.split()]
    assert vals == [ctypes.sizeof(ls.SgemmEntry), ctypes.sizeof(ls.DgemmEntry),
                    ls.SgemmEntry.M.offset, ls.SgemmEntry.alpha.offset,
                    ls.DgemmEntry.alpha.offset, ls.DgemmEntry.ldc.offset]
    s, d = ls.entry_dtypes()
    assert s.itemsize == vals[0] and d.itemsize == vals[1]
    assert s.fields["alpha"][1] == vals[3] and d.fields["alpha"][1] == vals[4]


def test_error_strings():
    for st in range(7):
        assert ls.error_string(st)
    assert ls.error_string(99) == "unknown status"


@pytest.mark.parametrize("args", [
    (2, 0, 8, 8, 8),    # bad transa
    (0, 5, 8, 8, 8),    # bad transb
    (0, 0, -1, 8, 8),   # negative M
    (0, 0, 8, 8, -3),   # negative K
])
def test_invalid_arguments_rejected_before_launch(args):
    ta, tb, M, N, K = args
    fake = 0x1000  # never dereferenced: validation fails first
    assert ls.sgemm(ta, tb, fake, fake, fake, M, N, K, check=False) == ls.ERR_INVALID_VALUE
    assert ls.dgemm(ta, tb, fake, fake, fake, M, N, K, check=False) == ls.ERR_INVALID_VALUE
    assert ls.sgemm_mp(ta, tb, fake, fake, fake, M, N, K, check=False) == ls.ERR_INVALID_VALUE


def test_null_pointers_rejected():
    assert ls.sgemm(0, 0, None, None, None, 4, 4, 4, check=False) == ls.ERR_INVALID_VALUE
    assert ls.sgemm_batched(None, 5, check=False) == ls.ERR_INVALID_VALUE
    assert ls.dgemm_batched(None, 5, check=False) == ls.ERR_INVALID_VALUE


def test_empty_problems_are_noops():
    # M == 0 or N == 0: nothing to compute, success without touching the device
    assert ls.sgemm(0, 0, None, None, None, 0, 5, 5, check=False) == ls.SUCCESS
    assert ls.dgemm(0, 1, None, None, None, 5, 0, 5, check=False) == ls.SUCCESS
    assert ls.sgemm_batched(None, 0, check=False) == ls.SUCCESS


def test_mode_setters_validate():
    assert ls.lib().LibShalom_set_precision(7) == ls.ERR_INVALID_VALUE
    assert ls.lib().LibShalom_set_splitk(-1) == ls.ERR_INVALID_VALUE
    ls.set_precision(ls.PREC_BF16X6)
    assert ls.get_precision() == ls.PREC_BF16X6
    ls.set_precision(ls.PREC_FP32)
    ls.lib().LibShalom_set_thread_ways(0, 4)
    assert ls.last_error() == ls.ERR_INVALID_VALUE
    ls.set_thread_nums(64)
    assert ls.last_error() == ls.SUCCESS
    ls.set_thread_nums(0)


def test_no_device_reported_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    fake = 0x1000
    st = ls.sgemm(0, 0, fake, fake, fake, 4, 4, 4, check=False)
    assert st == ls.ERR_NO_DEVICE


def test_host_calls_validate_before_device_work():
    import numpy as np
    a = np.zeros(64, np.float32)
    assert ls.sgemm_host(2, 0, a, a, a, 4, 4, 4, check=False) == ls.ERR_INVALID_VALUE
    assert ls.dgemm_host(0, 0, None, None, None, -1, 4, 4, check=False) == ls.ERR_INVALID_VALUE
    assert ls.sgemm_mp_host(0, 0, None, None, None, 4, 4, 4, check=False) == ls.ERR_INVALID_VALUE
    # M == 0: nothing to copy or compute
    assert ls.sgemm_host(0, 0, None, None, None, 0, 4, 4, check=False) == ls.SUCCESS
    # overlapping outputs of a batch cannot be copied back
    st = ls.sgemm_batched_strided_host(0, 4, 4, 4, 1.0, a, 16, a, 16, 0.0, a, 8, 2, check=False)
    assert st == ls.ERR_INVALID_VALUE


def test_host_pointer_of_arrays_and_cpu_tensors():
    import numpy as np
    a = np.zeros(8, np.float32)
    assert ls._hptr(a) == a.ctypes.data
    assert ls._hptr(None) is None and ls._hptr(1234) == 1234
    torch = pytest.importorskip("torch")
    t = torch.zeros(8)
    assert ls._hptr(t) == t.data_ptr()

    class DeviceTensor:  # stands in for a CUDA tensor on a machine without one
        is_cuda = True

        def data_ptr(self):
            return 0x1000
    with pytest.raises(ValueError):
        ls._hptr(DeviceTensor())


def test_convolution_arguments_validated():
    fake = 0x1000
    # kernel taller than the padded image, negative padding, zero stride
    assert ls.sconv2d_nchw(fake, 1, 1, 4, 4, fake, 1, 7, 3, 1, 1, 1, 1, fake,
                           check=False) == ls.ERR_INVALID_VALUE
    assert ls.sconv2d_nchw(fake, 1, 1, 4, 4, fake, 1, 3, 3, 1, 1, -1, 0, fake,
                           check=False) == ls.ERR_INVALID_VALUE
    assert ls.sconv2d_nchw(fake, 1, 1, 4, 4, fake, 1, 3, 3, 0, 1, 1, 1, fake,
                           check=False) == ls.ERR_INVALID_VALUE


def test_deferral_without_calls_and_invalid_calls():
    # an empty deferred section launches nothing; invalid calls are rejected
    # while deferring just as outside it
    ls.defer_begin()
    fake = 0x1000
    assert ls.sgemm(2, 0, fake, fake, fake, 4, 4, 4, check=False) == ls.ERR_INVALID_VALUE
    assert ls.dgemm(0, 0, None, None, None, 4, 4, 4, check=False) == ls.ERR_INVALID_VALUE
    assert ls.sgemm(0, 0, None, None, None, 0, 4, 4, check=False) == ls.SUCCESS
    assert ls.defer_pending() == 0
    assert ls.defer_flush(check=False) == ls.SUCCESS
