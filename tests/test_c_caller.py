"""The drop-in used the way the reference's own callers use it: a plain C
program (tests/c/hello_dropin.c, shaped like the reference's Hello.c and
benchmark/small_SGEMM/LibShalom_sgemm.c) that includes include/LibShalom.h,
links libshalom_b200.so and calls LibShalom_sgemm(NoTrans, Trans, ...) on
malloc'd HOST buffers.  The CPU test builds and links it; the GPU test runs
the 80^3 seed-0 call and compares C with the golden fixture the reference's
own SGEMM_NT instructions produced (bit-exact on rows >= 5, whose order is
k-sequential; the first row block's lane-split order within 1e-6)."""
import os
import subprocess

import numpy as np
import pytest

import libshalom_b200 as ls
from oracle import oracle as orc
from tests._util import normwise_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "hello_dropin.c")
FIXTURE = os.path.join(ROOT, "tests", "golden", "sgemm_nt_80_seed0.npz")


def _build(tmp_path):
    exe = tmp_path / "hello_dropin"
    libdir = os.path.dirname(ls.LIB_PATH)
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-std=c99", "-D_DEFAULT_SOURCE", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"), SRC, "-o", str(exe), "-L", libdir,
                    "-l:libshalom_b200.so", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
def test_c_caller_on_host_buffers_matches_reference_fixture(tmp_path):
    exe = _build(tmp_path)
    out = tmp_path / "C.bin"
    subprocess.run([str(exe), "0", str(out)], check=True, timeout=120)
    C = np.fromfile(out, np.float32).reshape(80, 80)
    Cref = np.load(FIXTURE)["C"]
    A, B = orc.gemm_inputs_f32(0, 80, 80, 80, 1)
    rows = np.arange(80) >= 5
    assert np.array_equal(C[rows], Cref[rows])
    assert normwise_err(C, Cref.astype(np.float64)) <= 1e-6
    assert np.array_equal(C, orc.sgemm_kseq(A, B, 1))  # this library's own order
