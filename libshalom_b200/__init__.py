"""Python host binding of the B200 LibShalom C ABI (``include/LibShalom.h``).

Every function here forwards to ``libshalom_b200.so`` through ctypes with
plain device pointers and sizes; there is no fallback: if the shared library
is missing or cannot be loaded, importing the compute entry points raises.
Torch tensors are accepted for convenience (their ``data_ptr()`` is passed);
torch is plumbing here (device memory, streams), not the compute path.

The reference interface mirrored here is ``NN_LIB/LibShalom.h:9-41``
(``LibShalom_sgemm``, ``LibShalom_sgemm_mp``, ``LibShalom_dgemm``,
``LibShalom_set_thread_nums``, ``LibShalom_set_thread_ways``).
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libshalom_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(_HERE), "include")

NoTrans = 0
Trans = 1
GEMM_K = 320
GEMM_N = 4096
GEMM_M = 256

SUCCESS = 0
ERR_INVALID_VALUE = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_NO_DEVICE = 4
ERR_ALLOC = 5
ERR_DEVICE_TIMEOUT = 6

PREC_FP32 = 0
PREC_BF16X3 = 1
PREC_BF16X6 = 2
DGEMM_FMA = 0
DGEMM_DMMA = 1
DGEMM_OZAKI = 2

# every symbol include/LibShalom.h declares
EXPORTED = (
    "LibShalom_sgemm", "LibShalom_sgemm_mp", "LibShalom_dgemm",
    "LibShalom_set_thread_nums", "LibShalom_set_thread_ways",
    "LibShalom_get_last_error", "LibShalom_error_string",
    "LibShalom_set_stream", "LibShalom_set_sync", "LibShalom_synchronize",
    "LibShalom_set_precision", "LibShalom_get_precision", "LibShalom_set_splitk",
    "LibShalom_set_dgemm_method", "LibShalom_get_dgemm_method",
    "LibShalom_set_tile_config", "LibShalom_set_autotune", "LibShalom_get_plan",
    "LibShalom_sgemm_ex", "LibShalom_dgemm_ex", "LibShalom_dgemm_stack", "LibShalom_sconv2d_nchw",
    "LibShalom_set_graph_cache",
    "LibShalom_set_tma",
    "LibShalom_finalize",
    "LibShalom_sgemm_batched", "LibShalom_sgemm_batched_strided",
    "LibShalom_dgemm_batched", "LibShalom_sgemm_mp_noalloc",
    "LibShalom_sgemm_host", "LibShalom_sgemm_mp_host", "LibShalom_dgemm_host",
    "LibShalom_sgemm_batched_strided_host",
    "LibShalom_defer_begin", "LibShalom_defer_flush", "LibShalom_defer_pending",
    "LibShalom_selftest_wait_expiry",
)

_L = ctypes.c_long
_I = ctypes.c_int
_P = ctypes.c_void_p
_F = ctypes.c_float


class SgemmEntry(ctypes.Structure):
    """LibShalom_sgemm_entry (64 bytes)."""
    _fields_ = [("A", _P), ("B", _P), ("C", _P),
                ("M", ctypes.c_int32), ("N", ctypes.c_int32), ("K", ctypes.c_int32),
                ("transb", ctypes.c_int32),
                ("lda", ctypes.c_int32), ("ldb", ctypes.c_int32), ("ldc", ctypes.c_int32),
                ("alpha", ctypes.c_float), ("beta", ctypes.c_float),
                ("reserved", ctypes.c_int32)]


class DgemmEntry(ctypes.Structure):
    """LibShalom_dgemm_entry (72 bytes)."""
    _fields_ = [("A", _P), ("B", _P), ("C", _P),
                ("M", ctypes.c_int32), ("N", ctypes.c_int32), ("K", ctypes.c_int32),
                ("transb", ctypes.c_int32),
                ("lda", ctypes.c_int32), ("ldb", ctypes.c_int32), ("ldc", ctypes.c_int32),
                ("reserved", ctypes.c_int32),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double)]


assert ctypes.sizeof(SgemmEntry) == 64 and ctypes.sizeof(DgemmEntry) == 72

_SIGS = {
    "LibShalom_sgemm": (None, [_I, _I, _P, _P, _P, _L, _L, _L]),
    "LibShalom_sgemm_mp": (None, [_I, _I, _P, _P, _P, _L, _L, _L]),
    "LibShalom_dgemm": (None, [_I, _I, _P, _P, _P, _L, _L, _L]),
    "LibShalom_set_thread_nums": (None, [_I]),
    "LibShalom_set_thread_ways": (None, [_I, _I]),
    "LibShalom_get_last_error": (_I, []),
    "LibShalom_error_string": (ctypes.c_char_p, [_I]),
    "LibShalom_set_stream": (_I, [_P]),
    "LibShalom_set_sync": (_I, [_I]),
    "LibShalom_synchronize": (_I, []),
    "LibShalom_set_precision": (_I, [_I]),
    "LibShalom_get_precision": (_I, []),
    "LibShalom_set_dgemm_method": (_I, [_I, _I]),
    "LibShalom_get_dgemm_method": (_I, []),
    "LibShalom_set_tile_config": (_I, [_I]),
    "LibShalom_set_autotune": (_I, [_I]),
    "LibShalom_get_plan": (_I, [ctypes.POINTER(ctypes.c_int)] * 3),
    "LibShalom_sgemm_ex": (_I, [_I, _I, _L, _L, _L, ctypes.c_float, _P, _L, _P, _L,
                                ctypes.c_float, _P, _L]),
    "LibShalom_dgemm_ex": (_I, [_I, _I, _L, _L, _L, ctypes.c_double, _P, _L, _P, _L,
                                ctypes.c_double, _P, _L]),
    "LibShalom_dgemm_stack": (_I, [_P, _L]),
    "LibShalom_set_graph_cache": (_I, [_I]),
    "LibShalom_sconv2d_nchw": (_I, [_P, _L, _L, _L, _L, _P, _L, _L, _L, _L, _L, _L, _L, _P]),
    "LibShalom_set_splitk": (_I, [_I]),
    "LibShalom_set_tma": (_I, [_I]),
    "LibShalom_finalize": (None, []),
    "LibShalom_selftest_wait_expiry": (_I, [_I]),
    "LibShalom_sgemm_batched": (_I, [_P, _L]),
    "LibShalom_sgemm_batched_strided": (_I, [_I, _L, _L, _L, _F, _P, _L, _P, _L, _F, _P, _L,
                                             _L]),
    "LibShalom_dgemm_batched": (_I, [_P, _L]),
    "LibShalom_sgemm_mp_noalloc": (_I, [_I, _I, _P, _P, _P, _L, _L, _L, _I]),
    "LibShalom_sgemm_host": (None, [_I, _I, _P, _P, _P, _L, _L, _L]),
    "LibShalom_sgemm_mp_host": (None, [_I, _I, _P, _P, _P, _L, _L, _L]),
    "LibShalom_dgemm_host": (None, [_I, _I, _P, _P, _P, _L, _L, _L]),
    "LibShalom_sgemm_batched_strided_host": (_I, [_I, _L, _L, _L, _F, _P, _L, _P, _L, _F, _P,
                                                  _L, _L]),
    "LibShalom_defer_begin": (_I, []),
    "LibShalom_defer_flush": (_I, []),
    "LibShalom_defer_pending": (_I, []),
}

_lib = None


class LibShalomError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {error_string(status)} (status {status})")


def lib() -> ctypes.CDLL:
    """The loaded C library.  Raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() "
                              "(make -C libshalom_b200/csrc)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def error_string(status: int) -> str:
    return lib().LibShalom_error_string(int(status)).decode()


def last_error() -> int:
    return lib().LibShalom_get_last_error()


def _ptr(x) -> int | None:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _hptr(x) -> int | None:
    """Host address of a numpy array or a CPU torch tensor (or an int)."""
    if x is None or isinstance(x, int):
        return x
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    if getattr(x, "is_cuda", False):
        raise ValueError("host-memory call given a CUDA tensor")
    return x.data_ptr()


def _check(status: int, what: str) -> None:
    if status != SUCCESS:
        raise LibShalomError(status, what)


# --------------------------------------------------------------------------
# drop-in entry points (void in C: status read back with get_last_error)
# --------------------------------------------------------------------------

def sgemm(transa, transb, C, A, B, M, N, K, check=True) -> int:
    lib().LibShalom_sgemm(transa, transb, _ptr(C), _ptr(A), _ptr(B), M, N, K)
    st = last_error()
    if check:
        _check(st, "LibShalom_sgemm")
    return st


def sgemm_mp(transa, transb, C, A, B, M, N, K, check=True) -> int:
    lib().LibShalom_sgemm_mp(transa, transb, _ptr(C), _ptr(A), _ptr(B), M, N, K)
    st = last_error()
    if check:
        _check(st, "LibShalom_sgemm_mp")
    return st


def dgemm(transa, transb, C, A, B, M, N, K, check=True) -> int:
    lib().LibShalom_dgemm(transa, transb, _ptr(C), _ptr(A), _ptr(B), M, N, K)
    st = last_error()
    if check:
        _check(st, "LibShalom_dgemm")
    return st


def sgemm_host(transa, transb, C, A, B, M, N, K, check=True) -> int:
    """LibShalom_sgemm with A, B and C in host memory (numpy / CPU tensors)."""
    lib().LibShalom_sgemm_host(transa, transb, _hptr(C), _hptr(A), _hptr(B), M, N, K)
    st = last_error()
    if check:
        _check(st, "LibShalom_sgemm_host")
    return st


def sgemm_mp_host(transa, transb, C, A, B, M, N, K, check=True) -> int:
    lib().LibShalom_sgemm_mp_host(transa, transb, _hptr(C), _hptr(A), _hptr(B), M, N, K)
    st = last_error()
    if check:
        _check(st, "LibShalom_sgemm_mp_host")
    return st


def dgemm_host(transa, transb, C, A, B, M, N, K, check=True) -> int:
    lib().LibShalom_dgemm_host(transa, transb, _hptr(C), _hptr(A), _hptr(B), M, N, K)
    st = last_error()
    if check:
        _check(st, "LibShalom_dgemm_host")
    return st


def defer_begin() -> None:
    """Record the following sgemm / sgemm_mp / dgemm calls in the host ring."""
    _check(lib().LibShalom_defer_begin(), "LibShalom_defer_begin")


def defer_flush(check=True) -> int:
    """Launch the recorded calls as grouped batches and end the deferral."""
    st = lib().LibShalom_defer_flush()
    if check:
        _check(st, "LibShalom_defer_flush")
    return st


def defer_pending() -> int:
    return lib().LibShalom_defer_pending()


def set_thread_nums(num: int) -> None:
    lib().LibShalom_set_thread_nums(int(num))


def set_thread_ways(tm: int, tn: int) -> None:
    lib().LibShalom_set_thread_ways(int(tm), int(tn))
    _check(last_error(), "LibShalom_set_thread_ways")


# --------------------------------------------------------------------------
# execution control
# --------------------------------------------------------------------------

def set_stream(stream) -> None:
    """stream: a torch.cuda.Stream, a raw cudaStream_t int, or None."""
    handle = None if stream is None else (stream if isinstance(stream, int)
                                          else stream.cuda_stream)
    _check(lib().LibShalom_set_stream(handle), "LibShalom_set_stream")


def set_sync(on: bool) -> None:
    _check(lib().LibShalom_set_sync(1 if on else 0), "LibShalom_set_sync")


def synchronize() -> None:
    _check(lib().LibShalom_synchronize(), "LibShalom_synchronize")


def set_precision(mode: int) -> None:
    _check(lib().LibShalom_set_precision(int(mode)), "LibShalom_set_precision")


def get_precision() -> int:
    return lib().LibShalom_get_precision()


def set_dgemm_method(method: int, slices: int = 0) -> None:
    """Arithmetic of dgemm_batched: DGEMM_FMA, DGEMM_DMMA or DGEMM_OZAKI
    (slices: INT8 digits per operand element, 4..9, 0 = 9)."""
    _check(lib().LibShalom_set_dgemm_method(int(method), int(slices)),
           "LibShalom_set_dgemm_method")


def get_dgemm_method() -> int:
    return lib().LibShalom_get_dgemm_method()


def set_tile_config(cfg: int) -> None:
    """Force a plain tile configuration (-1: measured table, then cost model)."""
    _check(lib().LibShalom_set_tile_config(int(cfg)), "LibShalom_set_tile_config")


def set_autotune(enable: bool) -> None:
    _check(lib().LibShalom_set_autotune(1 if enable else 0), "LibShalom_set_autotune")


def sgemm_ex(transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, check=True) -> int:
    """C = alpha op(A) op(B) + beta C with explicit leading dimensions (FP32)."""
    st = lib().LibShalom_sgemm_ex(transa, transb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb,
                                  beta, _ptr(C), ldc)
    if check:
        _check(st, "LibShalom_sgemm_ex")
    return st


def dgemm_ex(transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, check=True) -> int:
    """C = alpha op(A) op(B) + beta C with explicit leading dimensions (FP64)."""
    st = lib().LibShalom_dgemm_ex(transa, transb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb,
                                  beta, _ptr(C), ldc)
    if check:
        _check(st, "LibShalom_dgemm_ex")
    return st


class DgemmStack(ctypes.Structure):
    """LibShalom_dgemm_stack (host struct of device pointers)."""
    _fields_ = [("A_pool", ctypes.c_void_p), ("B_pool", ctypes.c_void_p),
                ("C_pool", ctypes.c_void_p), ("M", ctypes.c_void_p), ("N", ctypes.c_void_p),
                ("K", ctypes.c_void_p), ("m", ctypes.c_int32), ("n", ctypes.c_int32),
                ("k", ctypes.c_int32), ("transb", ctypes.c_int32), ("a_off", ctypes.c_void_p),
                ("b_off", ctypes.c_void_p), ("c_off", ctypes.c_void_p),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double)]


def dgemm_stack(A_pool, B_pool, C_pool, a_off, b_off, c_off, count, m=0, n=0, k=0, M=None,
                N=None, K=None, transb=0, alpha=1.0, beta=1.0, check=True) -> int:
    """Batched DGEMM from pools and per-product offsets (device arrays)."""
    st_ = DgemmStack(_ptr(A_pool), _ptr(B_pool), _ptr(C_pool),
                     _ptr(M) if M is not None else None, _ptr(N) if N is not None else None,
                     _ptr(K) if K is not None else None, m, n, k, transb,
                     _ptr(a_off), _ptr(b_off), _ptr(c_off), alpha, beta)
    st = lib().LibShalom_dgemm_stack(ctypes.byref(st_), count)
    if check:
        _check(st, "LibShalom_dgemm_stack")
    return st


def sconv2d_nchw(x, n, c, h, w, weights, oc, kh, kw, sh, sw, ph, pw, y, check=True) -> int:
    """FP32 NCHW convolution through im2col and the mp GEMM path."""
    st = lib().LibShalom_sconv2d_nchw(_ptr(x), n, c, h, w, _ptr(weights), oc, kh, kw, sh, sw,
                                      ph, pw, _ptr(y))
    if check:
        _check(st, "LibShalom_sconv2d_nchw")
    return st


def set_graph_cache(enable: bool) -> None:
    """Replay repeated identical single / mp calls from cached CUDA graphs."""
    _check(lib().LibShalom_set_graph_cache(1 if enable else 0), "LibShalom_set_graph_cache")


def get_plan():
    """(tile_config, splits, table_entries) of the last single / mp call."""
    c, s_, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().LibShalom_get_plan(ctypes.byref(c), ctypes.byref(s_), ctypes.byref(n))
    return c.value, s_.value, n.value


def set_splitk(splits: int) -> None:
    _check(lib().LibShalom_set_splitk(int(splits)), "LibShalom_set_splitk")


def set_tma(on: bool) -> None:
    """Tensor-core kernels: TMA warp-specialized variant (default) or cp.async."""
    _check(lib().LibShalom_set_tma(1 if on else 0), "LibShalom_set_tma")


def finalize() -> None:
    lib().LibShalom_finalize()


def selftest_wait_expiry(iterations: int = 0) -> int:
    """Runs the bounded-wait self-check kernel; returns its status
    (ERR_DEVICE_TIMEOUT is the expected outcome)."""
    return lib().LibShalom_selftest_wait_expiry(int(iterations))


# --------------------------------------------------------------------------
# batched entry points
# --------------------------------------------------------------------------

def sgemm_batched(entries_dev, count: int, check=True) -> int:
    """entries_dev: device buffer (tensor or pointer) of `count` SgemmEntry."""
    st = lib().LibShalom_sgemm_batched(_ptr(entries_dev), int(count))
    if check:
        _check(st, "LibShalom_sgemm_batched")
    return st


def sgemm_batched_strided(transb, M, N, K, alpha, A, strideA, B, strideB, beta, C, strideC,
                          count, check=True) -> int:
    st = lib().LibShalom_sgemm_batched_strided(transb, M, N, K, alpha, _ptr(A), strideA,
                                               _ptr(B), strideB, beta, _ptr(C), strideC, count)
    if check:
        _check(st, "LibShalom_sgemm_batched_strided")
    return st


def sgemm_batched_strided_host(transb, M, N, K, alpha, A, strideA, B, strideB, beta, C,
                               strideC, count, check=True) -> int:
    """Uniform batch with A, B and C in host memory (copies pipelined with the
    kernels; page-locked memory makes them asynchronous)."""
    st = lib().LibShalom_sgemm_batched_strided_host(transb, M, N, K, alpha, _hptr(A), strideA,
                                                    _hptr(B), strideB, beta, _hptr(C), strideC,
                                                    count)
    if check:
        _check(st, "LibShalom_sgemm_batched_strided_host")
    return st


def dgemm_batched(entries_dev, count: int, check=True) -> int:
    st = lib().LibShalom_dgemm_batched(_ptr(entries_dev), int(count))
    if check:
        _check(st, "LibShalom_dgemm_batched")
    return st


NOALLOC_SCRATCH_FLOATS = 2 * 1024 * 1024


def sgemm_mp_noalloc(transa, transb, C, A, B, M, N, K, splits, check=True) -> int:
    """LibShalom_sgemm_mp_noalloc: split-K SGEMM for callers that cannot
    allocate device memory; partial sums live in the library's fixed
    8 MiB device array (splits * M * N <= NOALLOC_SCRATCH_FLOATS)."""
    st = lib().LibShalom_sgemm_mp_noalloc(transa, transb, _ptr(C), _ptr(A), _ptr(B), M, N, K,
                                          int(splits))
    if check:
        _check(st, "LibShalom_sgemm_mp_noalloc")
    return st


def pack_entries(entries) -> bytes:
    """Serialise a list of SgemmEntry/DgemmEntry structures to bytes."""
    return b"".join(bytes(e) for e in entries)


# numpy views of the entry structures (for building large batches quickly)
def entry_dtypes():
    import numpy as np
    s = np.dtype([("A", "<u8"), ("B", "<u8"), ("C", "<u8"), ("M", "<i4"), ("N", "<i4"),
                  ("K", "<i4"), ("transb", "<i4"), ("lda", "<i4"), ("ldb", "<i4"),
                  ("ldc", "<i4"), ("alpha", "<f4"), ("beta", "<f4"), ("reserved", "<i4")])
    d = np.dtype([("A", "<u8"), ("B", "<u8"), ("C", "<u8"), ("M", "<i4"), ("N", "<i4"),
                  ("K", "<i4"), ("transb", "<i4"), ("lda", "<i4"), ("ldb", "<i4"),
                  ("ldc", "<i4"), ("reserved", "<i4"), ("alpha", "<f8"), ("beta", "<f8")])
    assert s.itemsize == 64 and d.itemsize == 72
    return s, d
