"""Autotuner of the single / mp GEMM schedulers.

For every shape class (kind, half-octaves of M, N and K) it times every
candidate schedule on the GPU -- tile configuration of the plain FP32 / FP64
kernels, split-K factor of the plain and tensor-core mp paths -- with CUDA
events (L2 flushed before every timed call, median of the repetitions), picks
the fastest, and writes

  csrc/ls_tune_table.inc   the table compiled into libshalom_b200.so
  a JSON report            every candidate's time, the cost model's own pick

Run on a B200, then rebuild (``make -C libshalom_b200/csrc``):

    python -m libshalom_b200.autotune --table libshalom_b200/csrc/ls_tune_table.inc \
        --report tune_report.json

``--evidence`` instead runs each irregular (mp) shape once with the table's
choice and once with the cost model's, for an ``ncu`` capture of both.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import libshalom_b200 as ls  # noqa: E402

KIND = {"s_single": 0, "s_mp": 1, "d_single": 2, "tc_bf16x3": 3, "tc_bf16x6": 4}

# shapes: the plain single-call sweep (cubes 8..128 and 80), the DGEMM block
# sizes, and irregular mp shapes (the six im2col / tall-skinny shapes plus a
# grid around them)
CUBES = list(range(8, 129, 8))
DCUBES = sorted(set(CUBES + [5, 9, 13, 22, 23, 26]))
IRREGULAR = [(64, 3136, 576), (128, 784, 1152), (256, 196, 2304), (512, 49, 4608),
             (20480, 32, 20480), (32, 20480, 4096)]
GRID = [(m, n, k) for m in (32, 128, 512, 2048, 8192) for n in (32, 196, 784, 4096)
        for k in (576, 2304, 8192)]


def half_octave(x: int) -> int:
    if x <= 1:
        return 0
    e = int(x).bit_length() - 1
    half = 1 if e >= 1 and x >= (3 << (e - 1)) else 0
    return min(127, 2 * e + half)


def shape_class(kind: str, M: int, N: int, K: int):
    return (KIND[kind], half_octave(M), half_octave(N), half_octave(K))


class Timer:
    def __init__(self, torch, reps):
        self.torch = torch
        self.reps = reps
        self.s = torch.cuda.Stream()
        torch.cuda.set_stream(self.s)
        ls.set_stream(self.s)
        ls.set_sync(False)
        # larger than the 126 MB L2
        self.flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")

    def __call__(self, fn):
        torch = self.torch
        fn()
        fn()
        self.s.synchronize()
        times = []
        for _ in range(self.reps):
            self.flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.s)
            fn()
            e1.record(self.s)
            self.s.synchronize()
            times.append(e0.elapsed_time(e1))
        return float(np.median(times))


def _operands(torch, M, N, K, dtype):
    A = torch.rand(M * K, device="cuda", dtype=dtype) * 2 - 1
    B = torch.rand(K * N, device="cuda", dtype=dtype) * 2 - 1
    C = torch.empty(M * N, device="cuda", dtype=dtype)
    return A, B, C


def _plan():
    return ls.get_plan()[:2]


def tune_shape(timer, torch, kind, M, N, K):
    """Times of every candidate {(cfg, splits): ms} and the model's pick."""
    dtype = torch.float64 if kind == "d_single" else torch.float32
    A, B, C = _operands(torch, M, N, K, dtype)
    if kind == "d_single":
        call = lambda: ls.dgemm(0, 0, C, A, B, M, N, K)  # noqa: E731
    elif kind == "s_single":
        call = lambda: ls.sgemm(0, 0, C, A, B, M, N, K)  # noqa: E731
    else:
        call = lambda: ls.sgemm_mp(0, 0, C, A, B, M, N, K)  # noqa: E731
    ls.set_precision({"tc_bf16x3": ls.PREC_BF16X3, "tc_bf16x6": ls.PREC_BF16X6}.get(
        kind, ls.PREC_FP32))
    ls.set_autotune(False)
    ls.set_tile_config(-1)
    ls.set_splitk(0)
    model_ms = timer(call)
    model = _plan()
    results = {}
    if kind in ("s_single", "d_single", "s_mp"):
        cfgs = range(4 if kind == "d_single" else 7)
    else:
        cfgs = [-1]
    splits = [1, 2, 4, 8, 16, 32] if kind == "s_mp" else (
        [1, 2, 3, 4, 6, 8, 9, 12, 16, 18, 24, 32, 36] if kind.startswith("tc") else [1])
    for cfg in cfgs:
        for sp in splits:
            ls.set_tile_config(cfg)
            ls.set_splitk(sp if kind != "s_single" and kind != "d_single" else 0)
            call()
            got = _plan()
            if got in results:
                continue  # the scheduler clamped this request to one already timed
            results[got] = timer(call)
    ls.set_tile_config(-1)
    ls.set_splitk(0)
    ls.set_autotune(True)
    ls.set_precision(ls.PREC_FP32)
    return results, model, model_ms


def run(args):
    import torch
    torch.cuda.set_device(0)
    timer = Timer(torch, args.reps)
    work = [("s_single", n, n, n) for n in CUBES + [80]]
    work += [("d_single", n, n, n) for n in DCUBES]
    mp = IRREGULAR + ([] if args.quick else GRID)
    for kind in ("s_mp", "tc_bf16x6", "tc_bf16x3"):
        work += [(kind, M, N, K) for (M, N, K) in mp]
    report = []
    for (kind, M, N, K) in work:
        res, model, model_ms = tune_shape(timer, torch, kind, M, N, K)
        best = min(res, key=res.get)
        report.append({"kind": kind, "M": M, "N": N, "K": K, "class": shape_class(kind, M, N, K),
                       "times_ms": {f"{c},{s}": t for (c, s), t in res.items()},
                       "best": list(best), "best_ms": res[best],
                       "model": list(model), "model_ms": model_ms})
        print(f"{kind:10s} {M:6d} {N:6d} {K:6d}  best cfg {best[0]:2d} splits {best[1]:2d} "
              f"{res[best]:8.4f} ms   model cfg {model[0]:2d} splits {model[1]:2d} "
              f"{model_ms:8.4f} ms", flush=True)
    # one choice per class: the candidate with the least summed time over the
    # class's shapes (only candidates every shape of the class timed)
    classes = {}
    for r in report:
        classes.setdefault(tuple(r["class"]), []).append(r)
    lines = ["// Generated by libshalom_b200/autotune.py on a B200; "
             "{kind, b(M), b(N), b(K), cfg, splits}"]
    for cls in sorted(classes):
        rs = classes[cls]
        common = set(rs[0]["times_ms"])
        for r in rs[1:]:
            common &= set(r["times_ms"])
        if not common:
            continue
        pick = min(common, key=lambda c: sum(r["times_ms"][c] for r in rs))
        cfg, sp = (int(v) for v in pick.split(","))
        gain = sum(r["model_ms"] for r in rs) / sum(r["times_ms"][pick] for r in rs)
        ex = ", ".join(f"{r['M']}x{r['N']}x{r['K']}" for r in rs[:3])
        lines.append(f"{{{cls[0]}, {cls[1]}, {cls[2]}, {cls[3]}, {cfg}, {max(sp, 0)}}},"
                     f"  // {ex}: {gain:.2f}x the cost model")
    with open(args.table, "w") as f:
        f.write("\n".join(lines) + "\n")
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    print(f"{len(lines) - 1} classes -> {args.table}")


def evidence(args):
    """Each irregular shape once with the table's choice, once with the model's
    (for an ncu capture of the pair)."""
    import torch
    torch.cuda.set_device(0)
    for prec in (ls.PREC_FP32, ls.PREC_BF16X6):
        ls.set_precision(prec)
        for (M, N, K) in IRREGULAR:
            A, B, C = _operands(torch, M, N, K, torch.float32)
            for tuned in (True, False):
                ls.set_autotune(tuned)
                ls.sgemm_mp(0, 0, C, A, B, M, N, K)
                torch.cuda.synchronize()
                print(f"prec {prec} {M}x{N}x{K} {'table' if tuned else 'model'} "
                      f"plan {ls.get_plan()[:2]}", flush=True)
    ls.set_autotune(True)
    ls.set_precision(ls.PREC_FP32)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--table", default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                    "csrc", "ls_tune_table.inc"))
    ap.add_argument("--report", default=None)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--quick", action="store_true", help="irregular shapes only, no grid")
    ap.add_argument("--evidence", action="store_true")
    args = ap.parse_args(argv)
    if args.evidence:
        evidence(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
