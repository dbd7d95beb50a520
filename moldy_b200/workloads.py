"""Seeded synthetic inputs for the MOLDY Fe EAM hot path.

All inputs are generated here (no dataset is involved).  The lattice follows
the reference's ``read_system`` conventions (``src/io_m.F90:73-256``):

* the box matrix B0 has the box vectors as columns, replicated n times;
* atoms are numbered with x replicas outermost, then y, then z, then the two
  bcc basis atoms (0,0,0) and (1/2,1/2,1/2);
* positions are fractional, never wrapped.

Displacements are Gaussian in Cartesian coordinates and converted with
B0^-1.  Velocities are Maxwell-Boltzmann (the reference's ``setvel`` draws
uniform components, ``src/thermostat_m.F90:201-249``), with the centre-of-mass
motion removed and the kinetic energy scaled to 1.5 (N-1) k T as ``setvel``
does with ``rqke`` (``src/thermostat_m.F90:94-99``).  They are stored as
x1 = B0^-1 v dt.  Box velocities start at zero.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import units
from .potentials import FE_FE, FeFeCoefficients

A0_FE = 2.8665          # bcc Fe lattice parameter (A)
RCUT_FETM = 6.0         # "range" returned by the FETRANSMETAL module (src/fetransmetal.F90:589-593)


@dataclasses.dataclass
class Workload:
    name: str
    nm: int
    x0: np.ndarray            # (nm, 3) fractional positions
    x1: np.ndarray            # (nm, 3) fractional velocity * dt
    x2: np.ndarray            # (nm, 3) fractional acceleration * dt^2 / 2
    b0: np.ndarray            # (3, 3) box, columns are box vectors (A)
    b1: np.ndarray
    b2: np.ndarray
    atomic_number: np.ndarray
    atomic_mass: np.ndarray
    del2: np.ndarray
    tgid: np.ndarray
    ivol: int
    ntcm: int
    ntc: int
    nnbrs: int
    atomstress: int
    rnear: float
    deltat: float             # model time units
    press: float              # model pressure units
    bdel2: float
    nlc: tuple
    coeffs: FeFeCoefficients
    meta: dict

    def copy(self) -> "Workload":
        w = dataclasses.replace(self)
        for f in ("x0", "x1", "x2", "b0", "b1", "b2", "atomic_number", "atomic_mass",
                  "del2", "tgid"):
            setattr(w, f, np.array(getattr(self, f), copy=True))
        w.meta = dict(self.meta)
        return w


def bcc_fractional(n: int) -> np.ndarray:
    """Fractional bcc positions of an n x n x n supercell in read_system order."""
    idx = np.arange(n, dtype=np.float64)
    i, j, k = np.meshgrid(idx, idx, idx, indexing="ij")
    cells = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)       # x outer, z inner
    basis = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]])
    pos = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)
    return pos / float(n)


def link_cell_counts(b0: np.ndarray, rnear: float) -> tuple:
    """nlc = max(3, int(B0(d,d) / rnear)) from the diagonal only (src/moldin.F90:252-257)."""
    return tuple(max(3, int(b0[d, d] / rnear)) for d in range(3))


def make_workload(n: int, *, a0: float = A0_FE, sigma: float = 0.05,
                  temperature: float = 300.0, ivol: int = 1, press_gpa: float = 0.0,
                  boxmass: float = 50.0, dt_fs: float = 1.0, rpad: float = 0.3,
                  nbrupdate: int = 100, nnbrs: int = 150, seed: int = 1234,
                  strain: np.ndarray | None = None, atomstress: int = 0,
                  coeffs: FeFeCoefficients = FE_FE, name: str | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    nm = 2 * n ** 3
    b0 = np.eye(3) * (a0 * n)
    if strain is not None:
        b0 = (np.eye(3) + np.asarray(strain, dtype=np.float64)) @ b0
    binv = np.linalg.inv(b0)
    x0 = bcc_fractional(n)
    if sigma > 0.0:
        disp = rng.normal(0.0, sigma, size=(nm, 3))
        x0 = x0 + disp @ binv.T
    mass = np.full(nm, units.FE_MASS)
    deltat = dt_fs * units.FS_TO_TIME
    x1 = np.zeros((nm, 3))
    if temperature > 0.0:
        v = rng.normal(0.0, 1.0, size=(nm, 3)) * np.sqrt(units.BK * temperature / mass)[:, None]
        v -= (mass[:, None] * v).sum(axis=0) / mass.sum()
        ke = 0.5 * float((mass[:, None] * v * v).sum())
        rqke = 1.5 * units.BK * temperature * (nm - 1)
        v *= math.sqrt(rqke / ke)
        x1 = (v * deltat) @ binv.T
    del2 = np.where(mass > 0.01, deltat * deltat / (2.0 * mass), 0.0)
    bmass = nm * boxmass
    bdel2 = deltat * deltat / (2.0 * bmass)
    rnear = RCUT_FETM + rpad
    return Workload(
        name=name or f"bcc_fe_{n}^3",
        nm=nm, x0=x0, x1=x1, x2=np.zeros((nm, 3)),
        b0=b0, b1=np.zeros((3, 3)), b2=np.zeros((3, 3)),
        atomic_number=np.full(nm, 26, dtype=np.int32), atomic_mass=mass, del2=del2,
        tgid=np.zeros((3, 3)), ivol=ivol, ntcm=nbrupdate, ntc=0, nnbrs=nnbrs,
        atomstress=atomstress, rnear=rnear, deltat=deltat,
        press=press_gpa * units.GPA_TO_PRESS, bdel2=bdel2,
        nlc=link_cell_counts(b0, rnear), coeffs=coeffs,
        meta=dict(n=n, a0=a0, sigma=sigma, temperature=temperature, seed=seed,
                  dt_fs=dt_fs, boxmass=boxmass, press_gpa=press_gpa, rpad=rpad),
    )


def config_small_nve(seed: int = 1) -> Workload:
    """2000-atom bcc Fe, sigma 0.05 A, 300 K, NVE (ivol=1), dt 1 fs, nbrupdate 100."""
    return make_workload(10, sigma=0.05, temperature=300.0, ivol=1, nbrupdate=100, seed=seed,
                         name="bcc_fe_2000_nve_300K")


def config_large_npt(n: int = 100, seed: int = 2) -> Workload:
    """2,000,000-atom bcc Fe (n=100), sigma 0.05 A, 1200 K, Parrinello-Rahman NPT
    at 0 GPa (ivol=0), box mass 50 amu/atom, dt 1 fs, nbrupdate 100."""
    return make_workload(n, sigma=0.05, temperature=1200.0, ivol=0, press_gpa=0.0,
                         boxmass=50.0, nbrupdate=100, seed=seed,
                         name=f"bcc_fe_{2 * n ** 3}_npt_1200K")


def config_liquid(n: int = 80, seed: int = 5, temperature: float = 300.0) -> Workload:
    """1,024,000-atom bcc Fe (n=80) for the heating/melting run, NPT, nbrupdate 20."""
    return make_workload(n, sigma=0.05, temperature=temperature, ivol=0, press_gpa=0.0,
                         boxmass=50.0, nbrupdate=20, seed=seed,
                         name=f"bcc_fe_{2 * n ** 3}_liquid")


def random_symmetric_strain(rng: np.random.Generator, amplitude: float) -> np.ndarray:
    e = rng.uniform(-amplitude, amplitude, size=6)
    return np.array([[e[0], e[3], e[4]], [e[3], e[1], e[5]], [e[4], e[5], e[2]]])


K_EFF_FE = 5.0          # effective spring constant for thermal displacements (eV/A^2)


def config_adjoint(nconf: int = 256, n: int = 8, seed: int = 4,
                   t_range: tuple = (300.0, 1800.0), strain_amplitude: float = 0.03) -> list:
    """Force-matching set: nconf seeded bcc Fe configurations of 2 n^3 atoms
    (default 256 x 1024).  Each has a temperature uniform in t_range, Gaussian
    displacements with sigma = sqrt(k T / k_eff), k_eff = 5 eV/A^2, and a
    symmetric strain with components uniform in +/- strain_amplitude."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(nconf):
        t = float(rng.uniform(*t_range))
        sigma = math.sqrt(units.BK * t / K_EFF_FE)
        strain = random_symmetric_strain(rng, strain_amplitude)
        w = make_workload(n, sigma=sigma, temperature=0.0, ivol=1, nbrupdate=100,
                          seed=int(rng.integers(1 << 30)), strain=strain,
                          name=f"bcc_fe_{2 * n ** 3}_fm{c:03d}")
        w.meta.update(config_temperature=t, strain=strain)
        out.append(w)
    return out


def config_batch(nsys: int = 1024, seed: int = 3, n_range: tuple = (4, 16), sigma: float = 0.1,
                 strain_amplitude: float = 0.02) -> list:
    """Batched supercells: nsys bcc Fe systems of n^3 cells, n uniform in
    n_range (inclusive), each with a symmetric strain whose components are
    uniform in +/- strain_amplitude, Gaussian displacements sigma (A), at rest
    and at a fixed box (ivol = 1)."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(nsys):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        strain = random_symmetric_strain(rng, strain_amplitude)
        w = make_workload(n, sigma=sigma, temperature=0.0, ivol=1, nbrupdate=100,
                          seed=int(rng.integers(1 << 30)), strain=strain,
                          name=f"bcc_fe_{2 * n ** 3}_batch{c:04d}")
        w.meta.update(strain=strain)
        out.append(w)
    return out


class ReferenceRandom:
    """The reference's random number generator (src/random_m.F90): rstart
    seeds the 97-entry lagged table, rand1 returns the next number in [0, 1).
    The reference seeds it with rstart(97, 33, 21, 82) (src/moldin.F90:175)."""

    def __init__(self, i=97, j=33, k=21, l=82):
        u = [0.0] * 98
        for ii in range(1, 98):
            s, t = 0.0, 0.5
            for _ in range(24):
                m = ((i * j) % 179 * k) % 179
                i, j, k = j, k, m
                l = (53 * l + 1) % 169
                if (l * m) % 64 >= 32:
                    s = s + t
                t = 0.5 * t
            u[ii] = s
        self.u = u
        self.c = 362436.0 / 16777216.0
        self.cd = 7654321.0 / 16777216.0
        self.cm = 16777213.0 / 16777216.0
        self.iu, self.ju = 97, 33

    def rand1(self) -> float:
        u = self.u
        uni = u[self.iu] - u[self.ju]
        if uni < 0.0:
            uni = uni + 1.0
        u[self.iu] = uni
        self.iu -= 1
        if self.iu == 0:
            self.iu = 97
        self.ju -= 1
        if self.ju == 0:
            self.ju = 97
        self.c = self.c - self.cd
        if self.c < 0.0:
            self.c = self.c + self.cm
        uni = uni - self.c
        if uni < 0.0:
            uni = uni + 1.0
        return uni


def setvel_reference(w: Workload, temprq: float, rng: ReferenceRandom | None = None) -> Workload:
    """Initial velocities as the reference's setvel draws them
    (src/thermostat_m.F90:201-256, with rqke = 1.5 bk temprq (nm - 1) from
    src/thermostat_m.F90:97): uniform fractional components rand1() - 0.5 per
    movable atom, the mass-weighted mean removed, scaled to rqke.  Box
    velocities are only drawn for ivol >= 1 (not 4), which this does not do."""
    if w.ivol >= 1 and w.ivol != 4:
        raise ValueError("setvel_reference draws atom velocities only (ivol < 1 or ivol == 4)")
    rng = rng or ReferenceRandom()
    nm = w.nm
    x1 = np.zeros((nm, 3))
    mass = w.atomic_mass
    movable = (w.atomic_number != 0) & (mass >= 0.1)
    nmove = 0
    for i in range(nm):
        if not movable[i]:
            continue
        x1[i, 0] = rng.rand1() - 0.5
        x1[i, 1] = rng.rand1() - 0.5
        x1[i, 2] = rng.rand1() - 0.5
        nmove += 1
    sxyz = [0.0, 0.0, 0.0]
    for d in range(3):
        s = 0.0
        for i in range(nm):
            s = s + x1[i, d] * mass[i]
        sxyz[d] = s / nmove
    b0 = w.b0
    s3 = 0.0
    for i in range(nm):
        if not movable[i]:
            continue
        for d in range(3):
            x1[i, d] = x1[i, d] - sxyz[d] / mass[i]
        rx = b0[0, 0] * x1[i, 0] + b0[0, 1] * x1[i, 1] + b0[0, 2] * x1[i, 2]
        ry = b0[1, 0] * x1[i, 0] + b0[1, 1] * x1[i, 1] + b0[1, 2] * x1[i, 2]
        rz = b0[2, 0] * x1[i, 0] + b0[2, 1] * x1[i, 1] + b0[2, 2] * x1[i, 2]
        s3 = s3 + mass[i] * (rx * rx + ry * ry + rz * rz)
    ke = s3 / w.deltat ** 2 / 2.0
    rqke = 1.5 * units.BK * temprq * (nm - 1)
    frac = float(np.sqrt(np.float32(np.float32(nmove) / np.float32(nm))))
    scale = math.sqrt(rqke / ke) * frac
    w2 = w.copy()
    w2.x1 = x1 * scale
    w2.meta.update(temperature=temprq, velocities="setvel (rand1)")
    return w2


def read_system_positions(n: int, rng: ReferenceRandom, dsp: float = 0.0, b0=None,
                          basis=((0.0, 0.0, 0.0), (0.5, 0.5, 0.5))) -> np.ndarray:
    """Fractional positions as read_system builds them (src/io_m.F90:221-248):
    x0 = (rand1() - 1/2) dsp / B0(1,1) + (1/nt) (i0 + xb), three rand1 draws per
    atom whatever dsp is, atoms in x-outer, z-inner, basis-innermost order."""
    rt = 1.0 / n
    b = np.asarray(b0) if b0 is not None else np.eye(3)
    out = np.zeros((2 * n ** 3 if len(basis) == 2 else len(basis) * n ** 3, 3))
    l = 0
    for i0 in range(n):
        for j0 in range(n):
            for k0 in range(n):
                for xb, yb, zb in basis:
                    out[l, 0] = (rng.rand1() - 0.5) * dsp / b[0, 0] + rt * (i0 + xb)
                    out[l, 1] = (rng.rand1() - 0.5) * dsp / b[1, 1] + rt * (j0 + yb)
                    out[l, 2] = (rng.rand1() - 0.5) * dsp / b[2, 2] + rt * (k0 + zb)
                    l += 1
    return out
