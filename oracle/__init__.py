"""CPU oracle for the MOLDY EAM hot path -- TEST INFRASTRUCTURE ONLY.

A ctypes wrapper around ``oracle/libmoldy_oracle.so``, the plain-C FP64
restatement of the reference Fortran (gjackland/moldy, FETRANSMETAL build):

* ``src/fetransmetal.F90`` (Fe-Fe functions, set_up_m) and ``src/lookup_m.F90``
  (tables and linear interpolation) -> ``fetm.c``;
* ``src/linkcell_m.F90``, ``src/neighbourlist_m.F90``, ``src/dynamics_m.F90``
  (rhoset, force, energy_calc, update_therm_avs), ``src/potential_m.F90``
  (embed), ``src/thermostat_m.F90`` (kinten), ``src/quench_m.F90``
  (velocityverlet) and the ``src/moldin.F90`` step order -> ``md.c``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package; the product library never does.

Parity status: unpinned by reference-produced vectors.  No Fortran compiler is
available, and the reference's shipped golden outputs use another material
module (IRON_CARBON).  The restatement is pinned by known-answer properties of
the reference's own coefficient file (perfect-lattice energy and density, zero
lattice forces, force = -dE/dx) checked in ``tests/test_oracle.py``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmoldy_oracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_longlong)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "libmoldy_oracle.so"],
                       check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    vp = ctypes.c_void_p
    sig = {
        "orc_create": (vp, [ctypes.c_int] * 5 + [ctypes.c_double] * 4),
        "orc_destroy": (None, [vp]),
        "orc_set_threads": (None, [ctypes.c_int]),
        "orc_get_max_threads": (ctypes.c_int, []),
        "orc_set_fetm": (ctypes.c_int, [vp, ctypes.c_int, _D, _D, ctypes.c_int, _D, _D]),
        "orc_set_lookup": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
        "orc_set_iron_carbon": (ctypes.c_int, [vp]),
        "orc_set_tables": (ctypes.c_int, [vp, ctypes.c_int] + [ctypes.c_double] * 4 + [_D] * 6),
        "orc_get_tables": (None, [vp] + [_D] * 6),
        "orc_get_fetm_derived": (None, [vp, _D]),
        "orc_src": (ctypes.c_double, [vp, ctypes.c_int, ctypes.c_double]),
        "orc_lookup": (ctypes.c_double, [vp, ctypes.c_int, ctypes.c_double]),
        "orc_set_state": (None, [vp] + [_D] * 12 + [_I, _D, _D, _D]),
        "orc_get_state": (None, [vp] + [_D] * 13),
        "orc_get_forces": (None, [vp, _D, _D, _D]),
        "orc_get_density": (None, [vp, _D, _D, _D]),
        "orc_get_atomstress": (None, [vp, _D, _D, _D]),
        "orc_get_force_out": (None, [vp, _D]),
        "orc_set_ntc": (None, [vp, ctypes.c_int]),
        "orc_get_ntc": (ctypes.c_int, [vp]),
        "orc_set_nlc": (None, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "orc_get_nlc": (None, [vp, _I]),
        "orc_linkup": (None, [vp]),
        "orc_relink": (None, [vp]),
        "orc_get_linkcells": (None, [vp, _I, _I, _I]),
        "orc_update_neighbourlist": (ctypes.c_int, [vp]),
        "orc_get_nlist": (None, [vp, _I, _I]),
        "orc_force": (ctypes.c_int, [vp]),
        "orc_velocityverlet": (ctypes.c_int, [vp]),
        "orc_update_therm_avs": (None, [vp, _D]),
        "orc_energy_calc": (None, [vp, _D]),
        "orc_md_init": (ctypes.c_int, [vp]),
        "orc_md_step": (ctypes.c_int, [vp, _D]),
        "orc_quench": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _D]),
        "orc_set_thermostat": (None, [vp, ctypes.c_double, ctypes.c_double]),
        "orc_get_thermostat": (None, [vp, _D]),
        "orc_scalev": (None, [vp]),
        "orc_rdf": (None, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _I, ctypes.c_int, _L, _L, _L]),
        "orc_rdf_rneighbour": (None, [_L, _L, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]),
        "orc_ackland_jones": (None, [vp, ctypes.c_int, _I, ctypes.c_int, _D, _I, _I, _I]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _lp(a):
    return a.ctypes.data_as(_L)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_I)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    _load().orc_set_threads(int(n))


def max_threads() -> int:
    return int(_load().orc_get_max_threads())


class Oracle:
    """One simulated system held by the C oracle (reference module globals)."""

    def __init__(self, nm, *, nnbrs=150, ivol=1, ntcm=100, atomstress=0,
                 rnear=6.3, deltat=0.0982269, press=0.0, bdel2=0.0):
        lib = _load()
        self.nm = int(nm)
        self.nnbrs = int(nnbrs)
        self._h = lib.orc_create(self.nm, self.nnbrs, int(ivol), int(ntcm), int(atomstress),
                                 float(rnear), float(deltat), float(press), float(bdel2))
        if not self._h:
            raise ValueError("orc_create failed")
        self._lib = lib

    def close(self):
        if self._h:
            self._lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # potential ---------------------------------------------------------
    def set_fetm(self, av, rv, ap, rp):
        av, rv, ap, rp = (_f64(v) for v in (av, rv, ap, rp))
        st = self._lib.orc_set_fetm(self._h, len(av), _dp(av), _dp(rv), len(ap), _dp(ap), _dp(rp))
        if st:
            raise RuntimeError(f"orc_set_fetm status {st}")

    def set_iron_carbon(self):
        """Fe-Fe functions of the IRON_CARBON module (src/iron_carbon.F90)."""
        self._lib.orc_set_iron_carbon(self._h)

    def set_lookup(self, uselookup=True, nlookup=5000):
        st = self._lib.orc_set_lookup(self._h, int(bool(uselookup)), int(nlookup))
        if st:
            raise RuntimeError(f"orc_set_lookup status {st}")
        self.nlookup = int(nlookup)

    def set_tables(self, tables, rmin=0.0, rmax=6.0, rhomin=0.0, rhomax=10000.0):
        """A caller's own lookup_m tables (dict of vee, dvee, phi, dphi, emb,
        demb with nlookup + 1 nodes each) over [rmin, rmax] and [rhomin, rhomax]."""
        t = [_f64(tables[k]) for k in ("vee", "dvee", "phi", "dphi", "emb", "demb")]
        n = len(t[0]) - 1
        st = self._lib.orc_set_tables(self._h, n, float(rmin), float(rmax), float(rhomin), float(rhomax),
                                      *[_dp(a) for a in t])
        if st:
            raise RuntimeError(f"orc_set_tables status {st}")
        self.nlookup = n

    def tables(self):
        n = self.nlookup + 1
        t = [np.zeros(n) for _ in range(6)]
        self._lib.orc_get_tables(self._h, *[_dp(a) for a in t])
        return dict(zip(["vee", "dvee", "phi", "dphi", "emb", "demb"], t))

    def fetm_derived(self):
        o = np.zeros(8)
        self._lib.orc_get_fetm_derived(self._h, _dp(o))
        return dict(zip(["bier_cut1", "bier_cut2", "sc1", "sc2", "sc3", "sc4",
                         "phi_cut1", "phi_cut2"], o.tolist()))

    def src(self, which: int, r: float) -> float:
        return float(self._lib.orc_src(self._h, int(which), float(r)))

    def lookup(self, which: int, r: float) -> float:
        return float(self._lib.orc_lookup(self._h, int(which), float(r)))

    # state -------------------------------------------------------------
    def set_state(self, x0, x1, x2, b0, b1, b2, atomic_number, atomic_mass, del2, tgid=None):
        """x0/x1/x2 are (nm,3) arrays; b* are 3x3 (row i, column j) arrays."""
        x0, x1, x2 = (np.asarray(a, dtype=np.float64) for a in (x0, x1, x2))
        cols = [_f64(x0[:, 0]), _f64(x0[:, 1]), _f64(x0[:, 2]),
                _f64(x1[:, 0]), _f64(x1[:, 1]), _f64(x1[:, 2]),
                _f64(x2[:, 0]), _f64(x2[:, 1]), _f64(x2[:, 2])]
        mats = [_f64(np.asarray(m, dtype=np.float64).ravel(order="F")) for m in (b0, b1, b2)]
        zn = np.ascontiguousarray(atomic_number, dtype=np.int32)
        am = _f64(atomic_mass)
        d2 = _f64(del2)
        tg = None if tgid is None else _f64(np.asarray(tgid).ravel(order="F"))
        self._lib.orc_set_state(self._h, *[_dp(c) for c in cols], *[_dp(m) for m in mats],
                                _ip(zn), _dp(am), _dp(d2), _dp(tg))

    def get_state(self):
        n = self.nm
        cols = [np.zeros(n) for _ in range(9)]
        mats = [np.zeros(9) for _ in range(4)]
        self._lib.orc_get_state(self._h, *[_dp(c) for c in cols], *[_dp(m) for m in mats])
        x0 = np.stack(cols[0:3], axis=1)
        x1 = np.stack(cols[3:6], axis=1)
        x2 = np.stack(cols[6:9], axis=1)
        b0, b1, b2, tgid = (m.reshape(3, 3, order="F") for m in mats)
        return dict(x0=x0, x1=x1, x2=x2, b0=b0, b1=b1, b2=b2, tgid=tgid)

    def forces(self):
        f = [np.zeros(self.nm) for _ in range(3)]
        self._lib.orc_get_forces(self._h, *[_dp(a) for a in f])
        return np.stack(f, axis=1)

    def density(self):
        d = [np.zeros(self.nm) for _ in range(3)]
        self._lib.orc_get_density(self._h, *[_dp(a) for a in d])
        return dict(rho=d[0], afrho=d[1], dafrho=d[2])

    def atomstress(self):
        d = [np.zeros(self.nm) for _ in range(3)]
        self._lib.orc_get_atomstress(self._h, *[_dp(a) for a in d])
        return np.stack(d, axis=1)

    def force_out(self):
        o = np.zeros(65)
        self._lib.orc_get_force_out(self._h, _dp(o))
        names = ["tp", "tk", "tc", "tg", "tgdot", "tgid", "fb"]
        out = {"pe": float(o[0]), "vol": float(o[1])}
        for k, nme in enumerate(names):
            out[nme] = o[2 + 9 * k: 11 + 9 * k].reshape(3, 3, order="F")
        return out

    @property
    def ntc(self):
        return int(self._lib.orc_get_ntc(self._h))

    @ntc.setter
    def ntc(self, v):
        self._lib.orc_set_ntc(self._h, int(v))

    # link cells / neighbour list ---------------------------------------
    def set_nlc(self, nlcx, nlcy, nlcz):
        self._lib.orc_set_nlc(self._h, int(nlcx), int(nlcy), int(nlcz))
        self.ncell = int(nlcx) * int(nlcy) * int(nlcz)

    def linkup(self):
        self._lib.orc_linkup(self._h)

    def relink(self):
        self._lib.orc_relink(self._h)

    def linkcells(self):
        l0 = np.zeros(self.ncell, dtype=np.int32)
        link = np.zeros(self.nm, dtype=np.int32)
        ic = np.zeros(self.nm, dtype=np.int32)
        self._lib.orc_get_linkcells(self._h, _ip(l0), _ip(link), _ip(ic))
        return l0, link, ic

    def update_neighbourlist(self):
        return int(self._lib.orc_update_neighbourlist(self._h))

    def nlist(self):
        """Returns (nlist[nm, nnbrs] with 1-based entries, numn[nm])."""
        nl = np.zeros(self.nnbrs * self.nm, dtype=np.int32)
        nn = np.zeros(self.nm, dtype=np.int32)
        self._lib.orc_get_nlist(self._h, _ip(nl), _ip(nn))
        return nl.reshape(self.nm, self.nnbrs), nn

    # hot path ------------------------------------------------------------
    def force(self):
        st = self._lib.orc_force(self._h)
        if st:
            raise RuntimeError(f"oracle force status {st}")

    def velocityverlet(self):
        st = self._lib.orc_velocityverlet(self._h)
        if st:
            raise RuntimeError(f"oracle velocityverlet status {st}")

    def update_therm_avs(self):
        o = np.zeros(3)
        self._lib.orc_update_therm_avs(self._h, _dp(o))
        return o

    def energy_calc(self):
        e = np.zeros(self.nm)
        self._lib.orc_energy_calc(self._h, _dp(e))
        return e

    def md_init(self):
        st = self._lib.orc_md_init(self._h)
        if st:
            raise RuntimeError(f"oracle md_init status {st}")

    def md_step(self):
        o = np.zeros(12)
        st = self._lib.orc_md_step(self._h, _dp(o))
        if st:
            raise RuntimeError(f"oracle md_step status {st}")
        keys = ["ke", "pe", "te", "h", "th", "vol", "s1", "s2", "s3", "temp", "boxke", "ntc"]
        return dict(zip(keys, o.tolist()))

    def set_thermostat(self, nose, rqke):
        self._lib.orc_set_thermostat(self._h, float(nose), float(rqke))

    def thermostat(self):
        v = np.zeros(4)
        self._lib.orc_get_thermostat(self._h, _dp(v))
        return {"nose": v[0], "rqke": v[1], "snhv": v[2], "thermotimer": v[3]}

    def scalev(self):
        self._lib.orc_scalev(self._h)

    def quench(self, maxfn=1000, criterion=0, fmax=1e-4):
        """quench_m::quench (VA14CD + derivs).  criterion 0: the reference's
        gsumsq <= 5e-7 nm; 1: max real force <= fmax (eV/A)."""
        o = np.zeros(8)
        st = self._lib.orc_quench(self._h, int(maxfn), int(criterion), float(fmax), _dp(o))
        if st:
            raise RuntimeError(f"oracle quench status {st}")
        return _quench_dict(o)


    # analysis_m::rdf ------------------------------------------------------
    def _spec(self, spec):
        if spec is None:
            spec = np.zeros(self.nm, dtype=np.int32)
        return np.ascontiguousarray(spec, dtype=np.int32)

    def rdf(self, maxbin=500, binsperangstrom=50, mode=0, spec=None, nspec=1):
        """Pair histogram hist[ibin, si, sj] (ibin 0..maxbin), natoms per
        species and the count of pairs closer than 2 A.  mode 0: half-list
        pairs (the current routine); 1: every pair (its older form)."""
        sp = self._spec(spec)
        h = np.zeros((maxbin + 1) * nspec * nspec, dtype=np.int64)
        na = np.zeros(nspec, dtype=np.int64)
        nc = np.zeros(1, dtype=np.int64)
        self._lib.orc_rdf(self._h, int(mode), int(maxbin), int(binsperangstrom), _ip(sp), int(nspec), _lp(h),
                          _lp(na), _lp(nc))
        return {"hist": h.reshape(maxbin + 1, nspec, nspec), "natoms": na, "nclose": int(nc[0])}

    @staticmethod
    def rneighbour(hist, natoms, binsperangstrom=50):
        _load()
        h = np.ascontiguousarray(hist, dtype=np.int64)
        nspec = h.shape[1]
        rn = np.zeros(nspec * nspec)
        _lib.orc_rdf_rneighbour(_lp(h), _lp(np.ascontiguousarray(natoms, dtype=np.int64)), h.shape[0] - 1,
                                int(binsperangstrom), nspec, _dp(rn))
        return rn.reshape(nspec, nspec)

    def ackland_jones(self, rn, mode=0, spec=None):
        """Per-atom Ackland-Jones class (0 unknown, 1 bcc, 2 fcc, 3 hcp, 4
        icosahedral), coordination nn and the eight bond-angle counts chi."""
        sp = self._spec(spec)
        rn = np.ascontiguousarray(rn, dtype=np.float64)
        nspec = rn.shape[0]
        aj = np.zeros(self.nm, dtype=np.int32)
        nn = np.zeros(self.nm, dtype=np.int32)
        chi = np.zeros(8 * self.nm, dtype=np.int32)
        self._lib.orc_ackland_jones(self._h, int(mode), _ip(sp), nspec, _dp(rn), _ip(aj), _ip(nn), _ip(chi))
        return {"aj": aj, "nn": nn, "chi": chi.reshape(self.nm, 8)}


def _quench_dict(o8):
    keys = ["f", "pe", "gsumsq", "fmax", "nfev", "iterations", "iflag", "status"]
    d = dict(zip(keys, o8.tolist()))
    for k in ("nfev", "iterations", "iflag", "status"):
        d[k] = int(d[k])
    return d


def from_workload(w, *, uselookup=True, nlookup=5000, threads=None) -> Oracle:
    """Builds an oracle system from a :class:`moldy_b200.workloads.Workload`."""
    if threads is not None:
        set_threads(threads)
    o = Oracle(w.nm, nnbrs=w.nnbrs, ivol=w.ivol, ntcm=w.ntcm, atomstress=w.atomstress,
               rnear=w.rnear, deltat=w.deltat, press=w.press, bdel2=w.bdel2)
    c = w.coeffs
    o.set_fetm(c.av, c.rv, c.ap, c.rp)
    o.set_lookup(uselookup, nlookup)
    o.set_state(w.x0, w.x1, w.x2, w.b0, w.b1, w.b2, w.atomic_number, w.atomic_mass, w.del2,
                w.tgid)
    o.set_nlc(*w.nlc)
    o.ntc = w.ntc
    o.linkup()
    return o
