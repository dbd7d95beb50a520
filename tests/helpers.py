"""Shared helpers for the parity tests: run the oracle and the GPU library on
the same seeded inputs and compare with written tolerances."""
from __future__ import annotations

import numpy as np


def real_forces(f_frac: np.ndarray, b0: np.ndarray) -> np.ndarray:
    """Real forces B0 f in eV/A (src/dynamics_m.F90:603-606)."""
    return f_frac @ np.asarray(b0).T


def rel_norm_err(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / max(||b||, tiny): a norm-wise relative error."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / max(nb, 1e-300))


def pair_set(nlist: np.ndarray, numn: np.ndarray) -> set:
    """Unordered pair set of a half list (1-based entries)."""
    s = set()
    for i in range(len(numn)):
        for j in nlist[i, :numn[i]]:
            a, b = i + 1, int(j)
            s.add((a, b) if a < b else (b, a))
    return s


def perturb(w, rng, amp_frac: float):
    """Random fractional displacements (uniform, +/- amp_frac) of a workload copy."""
    w2 = w.copy()
    w2.x0 = w2.x0 + rng.uniform(-amp_frac, amp_frac, size=w2.x0.shape)
    return w2
