"""Shared helpers of the test-suite (device buffers, error metrics)."""
from __future__ import annotations

import numpy as np


def to_dev(a: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def to_host(t) -> np.ndarray:
    return t.detach().cpu().numpy()


def normwise_err(C: np.ndarray, ref: np.ndarray) -> float:
    """max|C - ref| / max|ref| (0 when both are zero)."""
    d = np.max(np.abs(C.astype(np.float64) - ref)) if C.size else 0.0
    m = np.max(np.abs(ref)) if ref.size else 0.0
    if m == 0.0:
        return float(d)
    return float(d / m)


def componentwise_err(C: np.ndarray, ref: np.ndarray, absprod: np.ndarray) -> float:
    """max |C - ref|_ij / (|A||B|)_ij over entries with a nonzero bound."""
    d = np.abs(C.astype(np.float64) - ref)
    mask = absprod > 0
    if not mask.any():
        return float(np.max(d)) if d.size else 0.0
    return float(np.max(d[mask] / absprod[mask]))


def fp32_bound(K: int) -> float:
    """Deterministic FP32 bound for a K-term FMA chain, relative to (|A||B|)_ij:
    gamma_K = K u / (1 - K u), u = 2^-24 (Higham, Accuracy and Stability of
    Numerical Algorithms, eq. 3.5)."""
    u = 2.0 ** -24
    k = max(int(K), 1)
    return k * u / (1 - k * u)
