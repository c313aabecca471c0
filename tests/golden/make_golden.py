#!/usr/bin/env python3
"""Generates the golden fixtures of tests/golden/ by EXECUTING THE REFERENCE.

The reference's kernels are AArch64 NEON assembly inside C functions
(NN_LIB/test_SMM_NT.c, test_temp.c, test_temp_L1.c, DGEMM_NN.c).  This script
runs their instruction text on the AArch64 interpreter oracle/neon_emu.py,
with inputs from the reference benchmarks' own generator (random_matrix():
srand48(seed), a = 2.0*(float)drand48() - 1.0; restated bit-exactly in
oracle/oracle.c and checked against glibc), and stores the outputs.

Run where the reference source is checked out:
    python tests/golden/make_golden.py <reference checkout>
Nothing at test or bench time reads the reference; the tests regenerate the
inputs from the stored seeds and compare against the stored outputs.

Outputs
  sgemm_*.npz / dgemm_*.npz   one fixture per (kernel, shape, seed): C as the
                              reference computed it (NaN where it wrote nothing)
  dgemm_reference_behaviour.json   per (M % 7, N % 6) class of the DGEMM
                              workload sizes: elements the reference leaves
                              unwritten, values it gets wrong, and shapes on
                              which it reads through an unset register
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import neon_emu as emu  # noqa: E402
from oracle import oracle as orc  # noqa: E402

DGEMM_SIZES = [5, 9, 13, 16, 22, 23, 26, 32]


def save(name, **kw):
    np.savez_compressed(os.path.join(HERE, name), **kw)
    print("wrote", name, flush=True)


def ngm_nn_single_thread(nnlib, A, B, M, N, K):
    """LibShalom_sgemm_mp's N >> M driver (Small_NGM_NN_SGEMM,
    NN_LIB/SMM_NN_new.c:92-280) with one thread (T = Tm = Tn = 1), M <= GEMM_M:
    per GEMM_K = 320 block of K, the reference's own 8 x 12 micro-kernel SMM
    (NN_LIB/Kernel/SMM_m8n12_new.h:2846) over the N - N % 24 columns and its
    12 / 8 / 4 / 2 / 1-column edge kernels (SGEBP_NGM_NN, SMM_NN_new.c:8-88)
    run on the interpreter, with k_tag = the block's first k (0: store, else
    add into C) and m_tag = 0 (the kernels pack B as they go).  A is packed by
    NPACK (PACK.c:4) into [k][8 rows] blocks; that pass only moves data and is
    restated here as the transpose it is."""
    smm = os.path.join(nnlib, "Kernel", "SMM_m8n12_new.h")
    GK = 320
    C = np.full((M, N), np.nan, np.float32)
    Ac = np.zeros(K * M + 64, np.float32)
    for kk in range(0, K, GK):
        kc = min(GK, K - kk)
        for m0 in range(0, M, 8):
            mb = min(8, M - m0)
            Ac[kk * M + m0 * kc:kk * M + m0 * kc + kc * mb] = A[m0:m0 + mb, kk:kk + kc].T.ravel()
    Bc = np.zeros(N * GK + 64, np.float32)
    SSB = np.zeros(GK * 24 + 64, np.float32)
    Bf, Cf = np.ascontiguousarray(B).ravel(), C.ravel()
    n = 0
    for kk in range(0, K, GK):
        kc = min(GK, K - kk)
        edge = N % 24
        body = N - edge
        common = dict(M=M, K=kc, LN=N, LK=K, k_tag=kk, m_tag=0, id_tag=0)
        bufs = {"C": Cf, "A": Ac, "B": Bf, "Bc": Bc, "SB": SSB}
        if body:
            n += emu.run_asm(smm, "SMM", bufs, dict(common, N=body, stride_Bc=kc * 48),
                             {"A": kk * M, "B": kk * N})
        off = body
        for w, fn in ((12, "SMM"), (8, "SMM_NN_KERNEL8x8"), (4, "SMM_NN_KERNEL8x4"),
                      (2, "SMM_NN_KERNEL8x2"), (1, "SMM_NN_KERNEL8x1")):
            if edge >= w:
                extra = dict(stride_Bc=kc * 48) if fn == "SMM" else {}
                n += emu.run_asm(smm, fn, bufs, dict(common, N=w, **extra),
                                 {"C": off, "A": kk * M, "B": kk * N + off, "Bc": off * kc})
                edge -= w
                off += w
    return C, n


def main(ref_root):
    nnlib = os.path.join(ref_root, "NN_LIB")
    # LibShalom_sgemm_mp, N >> M (NGM) NN driver with its GEMM_K = 320 blocking
    # and k_tag accumulation; M a multiple of 8 as in the irregular shapes.
    # When a K block is not a multiple of 4 and N % 24 >= 12, the reference's
    # 12-column edge (the N == 12 packing path of SMM jumps past its K % 4
    # loop) drops the tail terms: edge_cols records those columns.
    for i, (M, N, K) in enumerate([(16, 96, 700), (8, 100, 333), (24, 60, 960), (32, 75, 1000),
                                   (16, 45, 500), (8, 39, 650), (40, 22, 333)]):
        seed = 300 + i
        A, B = orc.gemm_inputs_f32(seed, M, N, K, 0)
        C, n = ngm_nn_single_thread(nnlib, A, B, M, N, K)
        body = N - N % 24
        tail_blocks = any(min(320, K - kk) % 4 for kk in range(0, K, 320))
        edge = np.arange(body, body + 12) if (N % 24 >= 12 and tail_blocks) else np.arange(0)
        save(f"sgemm_mp_ngm_{M}x{N}x{K}_seed{seed}.npz", kind="sgemm_mp_ngm_ref",
             kernel="Small_NGM_NN_SGEMM (one thread)", M=M, N=N, K=K, seed=seed, C=C,
             edge_cols=edge, instructions=n)
    # config 1: LibShalom_sgemm(NoTrans, Trans), 80^3, seed 0 -> SGEMM_NT
    # config 2 NT shapes, seeds 16 + n/8
    for n, seed in [(80, 0), (16, 18), (48, 22)]:
        A, B = orc.gemm_inputs_f32(seed, n, n, n, 1)
        C = np.full((n, n), np.nan, np.float32)
        emu.run_kernel(os.path.join(nnlib, "test_SMM_NT.c"), "SGEMM_NT", A, B, C, n, n, n)
        save(f"sgemm_nt_{n}_seed{seed}.npz", kind="sgemm_nt_ref", kernel="SGEMM_NT",
             M=n, N=n, K=n, seed=seed, C=C)
    # config 2 NN shapes, seeds n/8: LibShalom_sgemm dispatches N > 96 to
    # SGEMM_NN (packed B strip) and N <= 96 to SGEMM_NN_L1 (NN_LIB/NN_SMM.c:10-20)
    for n in [8, 24, 40, 64, 96, 104, 128]:
        seed = n // 8
        A, B = orc.gemm_inputs_f32(seed, n, n, n, 0)
        C = np.full((n, n), np.nan, np.float32)
        if n > 96:
            emu.run_kernel(os.path.join(nnlib, "test_temp.c"), "SGEMM_NN", A, B, C, n, n, n,
                           sb_elems=n * 16 + 64)
            kernel = "SGEMM_NN"
        else:
            emu.run_kernel(os.path.join(nnlib, "test_temp_L1.c"), "SGEMM_NN_L1", A, B, C, n, n,
                           n)
            kernel = "SGEMM_NN_L1"
        save(f"sgemm_nn_{n}_seed{seed}.npz", kind="sgemm_nn_ref", kernel=kernel, M=n, N=n, K=n,
             seed=seed, C=C)

    # DGEMM_NN on the batched-DGEMM workload sizes
    behaviour = {}
    # shapes the reference computes fully and correctly (every M % 7, N % 6
    # class of the workload that it handles), plus two that show its defects:
    # (22, 16, 5) leaves row 21 unwritten, (23, 26, 13) gets the N2-tail
    # columns of its M2 row tail wrong
    fixtures = [(13, 32, 32), (9, 5, 13), (16, 13, 5), (26, 26, 13), (13, 23, 5),
                (26, 32, 32), (16, 16, 13), (23, 5, 32), (9, 32, 5), (26, 13, 13),
                (22, 16, 5), (23, 26, 13)]
    seed = 100
    for M in DGEMM_SIZES:
        for N in DGEMM_SIZES:
            for K in (5, 13, 32):
                seed += 1
                A, B = orc.dgemm_inputs(seed, M, N, K)
                C = np.full((M, N), np.nan)
                key = f"M%7={M % 7},N%6={N % 6}"
                b = behaviour.setdefault(key, {"shapes": 0, "faults": [], "unwritten_elements": 0,
                                               "wrong_values": 0})
                b["shapes"] += 1
                try:
                    emu.run_kernel(os.path.join(nnlib, "DGEMM_NN.c"), "DGEMM_NN", A, B, C, M, N, K)
                except IndexError as e:
                    b["faults"].append([M, N, K, str(e)])
                    continue
                exact = orc.dgemm_ld(A, B, 0)
                wrote = ~np.isnan(C)
                b["unwritten_elements"] += int((~wrote).sum())
                scale = np.abs(exact).max()
                b["wrong_values"] += int((wrote & (np.abs(C - exact) > 1e-12 * scale)).sum())
                if (M, N, K) in fixtures:
                    save(f"dgemm_nn_{M}x{N}x{K}_seed{seed}.npz", kind="dgemm_nn_ref",
                         kernel="DGEMM_NN", M=M, N=N, K=K, seed=seed, C=C)
    with open(os.path.join(HERE, "dgemm_reference_behaviour.json"), "w") as f:
        json.dump(behaviour, f, indent=1, sort_keys=True)
    print("wrote dgemm_reference_behaviour.json")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
