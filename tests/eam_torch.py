"""Test infrastructure: an FP64 torch restatement of one EAM force evaluation
in lookup mode, differentiable in the tables by torch autograd.

It gives the reference gradient the CUDA adjoint is checked against.  It
follows force() (src/dynamics_m.F90:135-401): rhoset over the half list (both
ends), embed (src/potential_m.F90:148-169, rho <= 1e-40 leaves an atom's
F and F' at zero), the pair loop with fp = -(DV + DP (F'_i + F'_j)) / r, and
the lookup_m interpolation (src/lookup_m.F90:307-394).  Outputs are the
quantities of write_energy_forces_stress (src/dynamics_m.F90:588-619):
E = pe, real forces F = B0 f, sigma(i,j) = -sum_k b0(j,k) tp(i,k) / vol.
The pair list comes from the oracle (1-based NLIST rows).
"""
from __future__ import annotations

import numpy as np
import torch

NAMES = ("vee", "dvee", "phi", "dphi", "emb", "demb")


def nint(x: np.ndarray) -> np.ndarray:
    """Fortran NINT: round half away from zero."""
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def half_pairs(nlist: np.ndarray, numn: np.ndarray):
    """(i, j) 0-based arrays of the half list, in list order."""
    nm = len(numn)
    mask = np.arange(nlist.shape[1])[None, :] < numn[:, None]
    i = np.repeat(np.arange(nm), numn)
    j = nlist[mask] - 1
    return i, j


def pair_vectors(x0: np.ndarray, b0: np.ndarray, i, j, ivol: int):
    """u = B0 (x_i - x_j) with the minimum-image convention of
    pr_get_realsep_from_dx (src/parrinellorahman_m.F90:149-173)."""
    d = x0[i] - x0[j]
    if ivol in (0, 1, 4):
        d = d - nint(d)
    elif ivol == 2:
        d[:, :2] = d[:, :2] - nint(d[:, :2])
    elif ivol == 5:
        d[:, 2] = d[:, 2] - nint(d[:, 2])
    return d @ b0.T


def interp(table: torch.Tensor, x: torch.Tensor, xmin: float, xmax: float, n: int) -> torch.Tensor:
    rng = xmax - xmin
    recipr, recipn, recips = 1.0 / rng, 1.0 / n, n / rng
    idx = torch.clamp(((n * (x - xmin)) * recipr).to(torch.int64), 0, n - 1)
    xlow = xmin + (rng * idx.to(torch.float64)) * recipn
    d = (x - xlow) * recips
    v = table[idx] * (1.0 - d) + table[idx + 1] * d
    return torch.where(x >= xmax, table[n].expand_as(x), v)


def eam_forward(x0, b0, i, j, mass, tables: dict, ranges=(0.0, 6.0, 0.0, 10000.0), ivol=1):
    """(E, F [nm,3], sigma [3,3]) as torch float64 tensors."""
    rmin, rmax, emin, emax = ranges
    n = tables["vee"].shape[0] - 1
    nm = x0.shape[0]
    u_np = pair_vectors(np.asarray(x0, dtype=np.float64), np.asarray(b0, dtype=np.float64), i, j, ivol)
    u = torch.as_tensor(u_np)
    r = torch.sqrt((u * u).sum(1))
    it, jt = torch.as_tensor(i), torch.as_tensor(j)
    ph = interp(tables["phi"], r, rmin, rmax, n)
    rho = torch.zeros(nm, dtype=torch.float64).index_add(0, it, ph).index_add(0, jt, ph)
    live = rho > 1e-40
    rho_safe = torch.where(live, rho, torch.ones_like(rho))
    em = torch.where(live, interp(tables["emb"], rho_safe, emin, emax, n), torch.zeros_like(rho))
    de = torch.where(live, interp(tables["demb"], rho_safe, emin, emax, n), torch.zeros_like(rho))
    v = interp(tables["vee"], r, rmin, rmax, n)
    dv = interp(tables["dvee"], r, rmin, rmax, n)
    dp = interp(tables["dphi"], r, rmin, rmax, n)
    e = v.sum() + em.sum()
    fp = -(dv + dp * (de[it] + de[jt])) / r
    fu = u * fp[:, None]
    f = torch.zeros(nm, 3, dtype=torch.float64).index_add(0, it, fu).index_add(0, jt, -fu)
    m = torch.as_tensor(np.asarray(mass, dtype=np.float64))
    keep = ((m[it] + m[jt]) > 0.1).to(torch.float64)
    vol = float(np.linalg.det(np.asarray(b0, dtype=np.float64)))
    sigma = -(u.T @ (u * (fp * keep)[:, None])) / vol
    return e, f, sigma


def torch_tables(tabs: dict, requires_grad=True) -> dict:
    return {k: torch.tensor(np.asarray(tabs[k], dtype=np.float64), requires_grad=requires_grad) for k in NAMES}
