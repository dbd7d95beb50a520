"""Radial distribution function and Ackland-Jones local structure of a
:class:`~moldy_b200.system.MoldySystem`'s current state, computed on the
device (analysis_m::rdf, src/analysis_m.F90:497-760), and the routine's
three output files.

``analyse(system)`` is the reference's ``call rdf(500, 50)`` at the end of a
run (src/moldin.F90:914-916): the pair histogram over the half neighbour list,
the fourth-neighbour radius of every species pair, the Ackland-Jones class of
every atom, and rdf.dat, prdf.dat and aj_b1f2h3.dat.  ``mode="all"`` bins
every pair of atoms instead, as the older form of the routine did when it
wrote the reference's shipped tests/reference/bcc_iron/rdf.dat.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import check

MODES = {"list": 0, "all": 1}
CLASSES = {0: "unknown", 1: "bcc", 2: "fcc", 3: "hcp", 4: "icosahedral"}


def _species(system, species, nspec):
    if species is None:
        return None, 1 if nspec is None else int(nspec)
    sp = np.ascontiguousarray(species, dtype=np.int32)
    if sp.shape != (system.nm,):
        raise ValueError("species needs one 0-based index per atom")
    return sp, int(sp.max()) + 1 if nspec is None else int(nspec)


def rdf(system, maxbin=500, binsperangstrom=50, mode="list", species=None, nspec=None) -> dict:
    """Pair histogram hist[ibin, si, sj] (ibin 0..maxbin, ibin = int(r *
    binsperangstrom)), the non-vacancy atoms of each species and the number
    of pairs closer than 2 A (the routine's warning)."""
    sp, ns = _species(system, species, nspec)
    L = _lib.load()
    h = np.zeros((maxbin + 1) * ns * ns, dtype=np.uint64)
    na = np.zeros(ns, dtype=np.int64)
    nc = ctypes.c_int64(0)
    check(L.moldy_gpu_rdf(system._h, MODES[mode], int(maxbin), int(binsperangstrom),
                          None if sp is None else sp.ctypes.data_as(_lib.I), ns,
                          h.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                          na.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(nc)))
    return {"hist": h.astype(np.int64).reshape(maxbin + 1, ns, ns), "natoms": na, "nclose": int(nc.value),
            "binsperangstrom": int(binsperangstrom)}


def rneighbour(hist, natoms, binsperangstrom=50) -> np.ndarray:
    """rnatoms(isp, jsp) (src/analysis_m.F90:619-637): for each species pair
    the radius of the bin at which the cumulative pair count first reaches
    4 min(natoms(isp), natoms(jsp)), in single precision as the reference
    writes it; rneighbour carries over between species pairs when the test
    never passes.  The reference sets isp <= jsp only; both orders get it."""
    hist = np.asarray(hist)
    maxbin = hist.shape[0] - 1
    ns = hist.shape[1]
    rn = np.zeros((ns, ns))
    rneighbour_ = 0.0
    for isp in range(ns):
        for jsp in range(isp, ns):
            irdf = hist[:, isp, jsp] + (hist[:, jsp, isp] if isp != jsp else 0)
            lim = 4 * min(int(natoms[isp]), int(natoms[jsp]))
            icount = 0
            for ibin in range(1, maxbin + 1):
                if icount < lim:
                    icount += int(irdf[ibin])
                    rneighbour_ = float(np.float32(ibin) / np.float32(binsperangstrom))
            rn[isp, jsp] = rn[jsp, isp] = rneighbour_
    return rn


def ackland_jones(system, rn, mode="list", species=None, with_chi=True) -> dict:
    """Per-atom Ackland-Jones class (0 unknown, 1 bcc, 2 fcc, 3 hcp, 4
    icosahedral), coordination nn within 1.45 rn^2 and the eight bond-angle
    counts chi (src/analysis_m.F90:644-757)."""
    rn = np.ascontiguousarray(np.atleast_2d(rn), dtype=np.float64)
    sp, ns = _species(system, species, rn.shape[0])
    L = _lib.load()
    aj = np.zeros(system.nm, dtype=np.int32)
    nn = np.zeros(system.nm, dtype=np.int32)
    chi = np.zeros(8 * system.nm, dtype=np.int32) if with_chi else None
    check(L.moldy_gpu_ackland_jones(system._h, MODES[mode], None if sp is None else sp.ctypes.data_as(_lib.I), ns,
                                    rn.ctypes.data_as(_lib.D), aj.ctypes.data_as(_lib.I),
                                    nn.ctypes.data_as(_lib.I), None if chi is None else chi.ctypes.data_as(_lib.I)))
    out = {"aj": aj, "nn": nn}
    if chi is not None:
        out["chi"] = chi.reshape(system.nm, 8)
    return out


# ------------------------------------------------------------ output files
def _radius(ibin, bpa):
    return np.float32(ibin) / np.float32(bpa)


def write_rdf(path, hist, binsperangstrom=50):
    """rdf.dat: '(F13.7,F18.7)' of r and n / r^2 per bin, single precision
    (src/analysis_m.F90:620-623)."""
    hist = np.asarray(hist)
    with open(path, "w") as f:
        for ibin in range(1, hist.shape[0]):
            r = _radius(ibin, binsperangstrom)
            n = np.float32(int(hist[ibin].sum()))
            f.write(f"{float(r):13.7f}{float(n / (r * r)):18.7f}\n")


def write_prdf(path, hist, binsperangstrom=50, labels=None):
    """prdf.dat: '(F13.7,F18.7,2I4)' per species pair isp <= jsp and bin
    (src/analysis_m.F90:625-634).  The reference's last two columns are
    atomic_index(isp) and atomic_index(jsp), the species of atoms number isp
    and jsp; labels[k] gives that number for k (default k + 1)."""
    hist = np.asarray(hist)
    ns = hist.shape[1]
    labels = list(range(1, ns + 1)) if labels is None else list(labels)
    with open(path, "w") as f:
        for isp in range(ns):
            for jsp in range(isp, ns):
                irdf = hist[:, isp, jsp] + (hist[:, jsp, isp] if isp != jsp else 0)
                for ibin in range(1, hist.shape[0]):
                    r = _radius(ibin, binsperangstrom)
                    v = np.float32(int(irdf[ibin])) / (r * r)
                    f.write(f"{float(r):13.7f}{float(v):18.7f}{labels[isp]:4d}{labels[jsp]:4d}\n")


def write_aj(path, aj, nn, znum):
    """aj_b1f2h3.dat: a title line and, per atom, its number, atomic number,
    class and coordination, in gfortran's list-directed layout
    (src/analysis_m.F90:616-617, 753)."""
    aj, nn, znum = (np.asarray(a) for a in (aj, nn, znum))
    with open(path, "w") as f:
        f.write(" atom        atomic number crystal structurecoordination\n")
        for i in range(len(aj)):
            f.write(f"{i + 1:12d}{int(znum[i]):12d}{int(aj[i]):12d}{int(nn[i]):12d}\n")


def analyse(system, maxbin=500, binsperangstrom=50, mode="list", species=None, znum=None, directory=None) -> dict:
    """The reference's rdf(maxbin, binsperangstrom): histogram, fourth-
    neighbour radii, Ackland-Jones classes; with ``directory`` also writes
    rdf.dat, prdf.dat and aj_b1f2h3.dat there.  znum: atomic number per atom
    for aj_b1f2h3.dat (default 26)."""
    h = rdf(system, maxbin, binsperangstrom, mode, species)
    rn = rneighbour(h["hist"], h["natoms"], binsperangstrom)
    a = ackland_jones(system, rn, mode, species)
    out = {**h, "rn": rn, **a}
    if directory is not None:
        os.makedirs(directory, exist_ok=True)
        write_rdf(os.path.join(directory, "rdf.dat"), h["hist"], binsperangstrom)
        sp = np.zeros(system.nm, dtype=np.int64) if species is None else np.asarray(species)
        ns = h["hist"].shape[1]
        labels = [int(sp[k]) + 1 if k < len(sp) else k + 1 for k in range(ns)]
        write_prdf(os.path.join(directory, "prdf.dat"), h["hist"], binsperangstrom, labels)
        z = np.full(system.nm, 26) if znum is None else znum
        write_aj(os.path.join(directory, "aj_b1f2h3.dat"), a["aj"], a["nn"], z)
    return out
