"""ctypes binding of oracle/liboracle.so -- TEST INFRASTRUCTURE ONLY.

The oracle is the checker for the parity tests, for ``__graft_entry__.smoke()``
and the timed CPU restatement of the reference for ``bench.py``'s
``cpu_baseline`` leg and ``--impl reference`` arm.  The shipped library never
imports it.  See ``oracle.c`` for which reference file:line each function
restates and for the parity status.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_L = ctypes.c_long
_U64 = ctypes.c_uint64
_D = ctypes.c_double
_I = ctypes.c_int


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        sig = {
            "orc_drand48": (None, [_U64, _U64, _L, _f64p]),
            "orc_fill_uniform_f32": (None, [_U64, _U64, _L, _f32p]),
            "orc_fill_uniform_f64": (None, [_U64, _U64, _L, _f64p]),
            "orc_fill_normal_scaled_f64": (None, [_U64, _U64, _L, _f64p, ctypes.c_void_p]),
            "orc_sgemm_f64": (None, [_I, _L, _L, _L, _D, _f32p, _L, _f32p, _L, _D,
                                      ctypes.c_void_p, _L, _f64p]),
            "orc_sgemm_absprod": (None, [_I, _L, _L, _L, _f32p, _L, _f32p, _L, _f64p]),
            "orc_dgemm_ld": (None, [_I, _L, _L, _L, _D, _f64p, _L, _f64p, _L, _D,
                                     ctypes.c_void_p, _L, _f64p]),
            "orc_sgemm_kseq": (None, [_I, _L, _L, _L, _f32p, _L, _f32p, _L, _f32p, _L, _L]),
            "orc_dgemm_kseq": (None, [_I, _L, _L, _L, _f64p, _L, _f64p, _L, _f64p, _L]),
            "orc_sgemm_nt_reforder": (None, [_L, _L, _L, _f32p, _f32p, _f32p]),
            "orc_dgemm_reforder": (None, [_L, _L, _L, _f64p, _f64p, _f64p]),
            "orc_port_sgemm": (None, [_I, _L, _L, _L, _f32p, _L, _f32p, _L, _f32p, _L]),
            "orc_port_dgemm": (None, [_L, _L, _L, _f64p, _L, _f64p, _L, _f64p, _L, _I]),
            "orc_port_sgemm_mp": (None, [_I, _L, _L, _L, _f32p, _f32p, _f32p, _I]),
            "orc_port_sgemm_batched": (None, [_L, _i32p, _i32p, _i32p, _i32p, _f32p, _f32p,
                                               _i64p, _f32p, _i64p, _f32p, _i64p, _I]),
            "orc_port_sgemm_strided": (None, [_I, _L, _L, _L, _L, _f32p, _f32p, _f32p, _I]),
            "orc_port_dgemm_batched": (None, [_L, _i32p, _i32p, _i32p, _f64p, _i64p, _f64p,
                                               _i64p, _f64p, _i64p, _I]),
            "orc_dgemm_batched_ld": (None, [_L, _i32p, _i32p, _i32p, _f64p, _i64p, _f64p,
                                             _i64p, _f64p, _i64p]),
            "orc_max_threads": (_I, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


# --------------------------------------------------------------------------
# generators
# --------------------------------------------------------------------------

def drand48(seed: int, n: int, skip: int = 0) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().orc_drand48(seed, skip, n, out)
    return out


def uniform_f32(seed: int, n: int, skip: int = 0) -> np.ndarray:
    """random_matrix() of the reference benchmarks: 2.0*(float)drand48()-1.0."""
    out = np.empty(n, np.float32)
    lib().orc_fill_uniform_f32(seed, skip, n, out)
    return out


def uniform_f64(seed: int, n: int, skip: int = 0) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().orc_fill_uniform_f64(seed, skip, n, out)
    return out


def normal_scaled_f64(seed: int, n: int, skip: int = 0) -> tuple[np.ndarray, float]:
    out = np.empty(n, np.float64)
    s = ctypes.c_double(0.0)
    lib().orc_fill_normal_scaled_f64(seed, skip, n, out, ctypes.byref(s))
    return out, s.value


def normal_scaled_draws(n: int) -> int:
    """drand48 draws consumed by one normal_scaled_f64 matrix of n entries."""
    return 1 + 2 * ((n + 1) // 2)


def gemm_inputs_f32(seed: int, M: int, N: int, K: int, transb: int):
    """A (M x K) then B (K x N, or N x K for transb) from one drand48 stream,
    as the reference benchmarks call random_matrix(M,K,A); random_matrix(K,N,B)."""
    A = uniform_f32(seed, M * K).reshape(M, K)
    B = uniform_f32(seed, K * N, skip=M * K)
    B = B.reshape(N, K) if transb else B.reshape(K, N)
    return A, B


def dgemm_inputs(seed: int, M: int, N: int, K: int):
    """A (M x K) then B (K x N), each normal(0,1) * 10^u with its own u in
    [-3, 3], from one drand48 stream (the batched-DGEMM workload's generator)."""
    A, _ = normal_scaled_f64(seed, M * K)
    B, _ = normal_scaled_f64(seed, K * N, skip=normal_scaled_draws(M * K))
    return A.reshape(M, K), B.reshape(K, N)


# --------------------------------------------------------------------------
# oracles
# --------------------------------------------------------------------------

def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def sgemm_f64(A, B, transb, alpha=1.0, beta=0.0, C=None, transa=0) -> np.ndarray:
    """alpha*op(A) op(B) + beta*C accumulated in double (FP32 inputs)."""
    A = _c(A.T if transa else A, np.float32)
    B = _c(B, np.float32)
    M, K = A.shape
    N = B.shape[0] if transb else B.shape[1]
    out = np.empty((M, N), np.float64)
    Cin = None
    if beta != 0.0:
        Cin = _c(C, np.float32)
    lib().orc_sgemm_f64(int(transb), M, N, K, alpha, A, K, B, B.shape[1], beta,
                        Cin.ctypes.data if Cin is not None else None, N, out)
    return out


def sgemm_absprod(A, B, transb, transa=0) -> np.ndarray:
    A = _c(A.T if transa else A, np.float32)
    B = _c(B, np.float32)
    M, K = A.shape
    N = B.shape[0] if transb else B.shape[1]
    out = np.empty((M, N), np.float64)
    lib().orc_sgemm_absprod(int(transb), M, N, K, A, K, B, B.shape[1], out)
    return out


def dgemm_ld(A, B, transb, alpha=1.0, beta=0.0, C=None, transa=0) -> np.ndarray:
    """FP64 oracle accumulated in x87 extended precision."""
    A = _c(A.T if transa else A, np.float64)
    B = _c(B, np.float64)
    M, K = A.shape
    N = B.shape[0] if transb else B.shape[1]
    out = np.empty((M, N), np.float64)
    Cin = _c(C, np.float64) if beta != 0.0 else None
    lib().orc_dgemm_ld(int(transb), M, N, K, alpha, A, K, B, B.shape[1], beta,
                       Cin.ctypes.data if Cin is not None else None, N, out)
    return out


def sgemm_kseq(A, B, transb, kblock=0, transa=0) -> np.ndarray:
    """FP32 k-sequential FMA chain per element (reference register-tile order);
    kblock=320 restates the mp drivers' GEMM_K blocking."""
    A = _c(A.T if transa else A, np.float32)
    B = _c(B, np.float32)
    M, K = A.shape
    N = B.shape[0] if transb else B.shape[1]
    out = np.empty((M, N), np.float32)
    lib().orc_sgemm_kseq(int(transb), M, N, K, A, K, B, B.shape[1], out, N, int(kblock))
    return out


def dgemm_kseq(A, B, transb, transa=0) -> np.ndarray:
    A = _c(A.T if transa else A, np.float64)
    B = _c(B, np.float64)
    M, K = A.shape
    N = B.shape[0] if transb else B.shape[1]
    out = np.empty((M, N), np.float64)
    lib().orc_dgemm_kseq(int(transb), M, N, K, A, K, B, B.shape[1], out, N)
    return out


def dgemm_reforder(A, B) -> np.ndarray:
    """DGEMM_NN's own rounding order (k-sequential, N1 tail lane-split)."""
    A = _c(A, np.float64)
    B = _c(B, np.float64)
    M, K = A.shape
    N = B.shape[1]
    out = np.empty((M, N), np.float64)
    lib().orc_dgemm_reforder(M, N, K, A, B, out)
    return out


def sgemm_nt_reforder(A, B) -> np.ndarray:
    """SGEMM_NT's own rounding order (lane-split rows 0..4 of each strip)."""
    A = _c(A, np.float32)
    B = _c(B, np.float32)
    M, K = A.shape
    N = B.shape[0]
    out = np.empty((M, N), np.float32)
    lib().orc_sgemm_nt_reforder(M, N, K, A, B, out)
    return out


# --------------------------------------------------------------------------
# CPU baseline port of the reference algorithm
# --------------------------------------------------------------------------

def port_sgemm(A, B, transb, C=None) -> np.ndarray:
    A = _c(A, np.float32)
    B = _c(B, np.float32)
    M, K = A.shape
    N = B.shape[0] if transb else B.shape[1]
    out = C if C is not None else np.empty((M, N), np.float32)
    lib().orc_port_sgemm(int(transb), M, N, K, A, K, B, B.shape[1], out, N)
    return out


def port_sgemm_mp(A, B, transb, threads: int, C=None) -> np.ndarray:
    A = _c(A, np.float32)
    B = _c(B, np.float32)
    M, K = A.shape
    N = B.shape[0] if transb else B.shape[1]
    out = C if C is not None else np.empty((M, N), np.float32)
    lib().orc_port_sgemm_mp(int(transb), M, N, K, A, B, out, int(threads))
    return out


def port_dgemm(A, B, C=None, accumulate=False) -> np.ndarray:
    A = _c(A, np.float64)
    B = _c(B, np.float64)
    M, K = A.shape
    N = B.shape[1]
    out = C if C is not None else np.zeros((M, N), np.float64)
    lib().orc_port_dgemm(M, N, K, A, K, B, N, out, N, int(accumulate))
    return out


def port_sgemm_strided(transb, M, N, K, count, A, B, C, threads: int):
    lib().orc_port_sgemm_strided(int(transb), M, N, K, count, A, B, C, int(threads))
    return C


def max_threads() -> int:
    return int(lib().orc_max_threads())
