"""Host-side mirror of the reference's hot-path call surface.

The reference (gjackland/moldy) drives its hot path through no-argument
Fortran routines acting on module globals.  :class:`MoldySystem` holds one
such set of globals on one GPU and exposes the same routines by name:

==========================  =============================================
method                      reference routine
==========================  =============================================
``set_up_fetm``             ``potential_set_lookup`` / ``potential_set_exact``
                            + ``set_up`` (src/potential_m.F90:181-280)
``linkup`` / ``relink``     src/linkcell_m.F90:122-274
``update_neighbourlist``    src/neighbourlist_m.F90:103-276
``force``                   src/dynamics_m.F90:135-401
``velocityverlet``          src/quench_m.F90:562-624
``update_therm_avs``        src/dynamics_m.F90:649-734
``energy_calc``             src/dynamics_m.F90:412-483
``md_init`` / ``md_steps``  the strain-loop preparation and mdloop of
                            src/moldin.F90:445-477, 575-791
==========================  =============================================

Every call goes through ``libmoldy_gpu.so``; errors come back as
:class:`moldy_b200._lib.MoldyError` with the reference's stop message.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_lib.D)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_lib.I)


def _mat_f(m):
    """3x3 (row i, column j) -> Fortran column-major 9-vector."""
    return None if m is None else _f64(np.asarray(m, dtype=np.float64).reshape(3, 3).ravel(order="F"))


def _mat_from_f(v):
    return np.asarray(v, dtype=np.float64).reshape(3, 3, order="F")


class MoldySystem:
    """One simulated system resident on one GPU."""

    def __init__(self, nm, *, rnear=6.3, deltat=0.0982269, press=0.0, bdel2=0.0, nnbrs=150,
                 ivol=1, ntcm=100, ntc=0, nlc=(0, 0, 0), atomstress=0, precision="fp64",
                 device=0):
        self._L = _lib.load()
        p = _lib.Params()
        p.rnear, p.deltat, p.press, p.bdel2 = float(rnear), float(deltat), float(press), float(bdel2)
        p.nm, p.nnbrs, p.ivol, p.ntcm, p.ntc = int(nm), int(nnbrs), int(ivol), int(ntcm), int(ntc)
        p.nlcx, p.nlcy, p.nlcz = (int(v) for v in nlc)
        p.atomstress = int(atomstress)
        p.precision = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
        p.device = int(device)
        h = _lib.H()
        check(self._L.moldy_gpu_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.nm = int(nm)
        self.nnbrs = int(nnbrs)
        self.params = p

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._L.moldy_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @classmethod
    def from_workload(cls, w, *, uselookup=True, nlookup=5000, precision="fp64", device=0):
        s = cls(w.nm, rnear=w.rnear, deltat=w.deltat, press=w.press, bdel2=w.bdel2,
                nnbrs=w.nnbrs, ivol=w.ivol, ntcm=w.ntcm, ntc=w.ntc, nlc=w.nlc,
                atomstress=w.atomstress, precision=precision, device=device)
        s.set_up_fetm(w.coeffs, uselookup=uselookup, nlookup=nlookup)
        s.set_state(w.x0, w.x1, w.x2, w.b0, w.b1, w.b2, w.atomic_number, w.atomic_mass, w.del2,
                    w.tgid)
        return s

    # ------------------------------------------------------------ potential
    def set_up_fetm(self, coeffs, *, uselookup=True, nlookup=5000):
        av, rv, ap, rp = (_f64(v) for v in (coeffs.av, coeffs.rv, coeffs.ap, coeffs.rp))
        check(self._L.moldy_gpu_set_fetm_fe(self._h, len(av), _dp(av), _dp(rv), len(ap), _dp(ap),
                                            _dp(rp), int(bool(uselookup)), int(nlookup)))
        self.nlookup = int(nlookup)
        self.n_knots = (len(av), len(ap))

    def set_up_iron_carbon(self, *, nlookup=5000):
        """Fe-Fe functions of the IRON_CARBON module, lookup tables."""
        check(self._L.moldy_gpu_set_iron_carbon_fe(self._h, int(nlookup)))
        self.nlookup = int(nlookup)

    def set_tables(self, tables: dict, *, rmin=0.0, rmax=6.0, rhomin=0.0, rhomax=10000.0):
        t = {k: _f64(tables[k]) for k in ("vee", "dvee", "phi", "dphi", "emb", "demb")}
        n = len(t["vee"]) - 1
        check(self._L.moldy_gpu_set_tables(self._h, n, rmin, rmax, rhomin, rhomax,
                                           *[_dp(t[k]) for k in ("vee", "dvee", "phi", "dphi",
                                                                 "emb", "demb")]))
        self.nlookup = n

    def tables(self) -> dict:
        n = self.nlookup + 1
        t = [np.zeros(n) for _ in range(6)]
        check(self._L.moldy_gpu_get_tables(self._h, *[_dp(a) for a in t]))
        return dict(zip(["vee", "dvee", "phi", "dphi", "emb", "demb"], t))

    # ---------------------------------------------------------------- state
    def set_state(self, x0=None, x1=None, x2=None, b0=None, b1=None, b2=None,
                  atomic_number=None, atomic_mass=None, del2=None, tgid=None):
        cols = []
        for arr in (x0, x1, x2):
            if arr is None:
                cols += [None, None, None]
            else:
                a = np.asarray(arr, dtype=np.float64)
                cols += [_f64(a[:, 0]), _f64(a[:, 1]), _f64(a[:, 2])]
        mats = [_mat_f(m) for m in (b0, b1, b2)]
        zn = None if atomic_number is None else np.ascontiguousarray(atomic_number, dtype=np.int32)
        am = None if atomic_mass is None else _f64(atomic_mass)
        d2 = None if del2 is None else _f64(del2)
        tg = _mat_f(tgid)
        check(self._L.moldy_gpu_set_state(self._h, *[_dp(c) for c in cols],
                                          *[_dp(m) for m in mats], _ip(zn), _dp(am), _dp(d2),
                                          _dp(tg)))

    def set_state_soa(self, x0, y0, z0, x1, y1, z1, x2, y2, z2, b0=None, b1=None, b2=None):
        """Uploads positions/velocities/accelerations from nine contiguous FP64
        arrays without copying them on the host (pinned buffers stay pinned)."""
        arrs = [np.asarray(a) for a in (x0, y0, z0, x1, y1, z1, x2, y2, z2)]
        for a in arrs:
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != (self.nm,):
                raise ValueError("set_state_soa needs contiguous float64 arrays of length nm")
        mats = [_mat_f(m) for m in (b0, b1, b2)]
        check(self._L.moldy_gpu_set_state(self._h, *[_dp(a) for a in arrs], *[_dp(m) for m in mats],
                                          None, None, None, None))

    def get_state_soa(self, out: list, forces: list | None = None):
        """Downloads x0..z2 into nine preallocated contiguous FP64 arrays (and the
        forces into three more) without intermediate host copies."""
        check(self._L.moldy_gpu_get_state(self._h, *[_dp(a) for a in out], None, None, None, None))
        if forces is not None:
            check(self._L.moldy_gpu_get_forces(self._h, *[_dp(a) for a in forces]))

    def get_state(self) -> dict:
        n = self.nm
        cols = [np.zeros(n) for _ in range(9)]
        mats = [np.zeros(9) for _ in range(4)]
        check(self._L.moldy_gpu_get_state(self._h, *[_dp(c) for c in cols],
                                          *[_dp(m) for m in mats]))
        return dict(x0=np.stack(cols[0:3], 1), x1=np.stack(cols[3:6], 1), x2=np.stack(cols[6:9], 1),
                    b0=_mat_from_f(mats[0]), b1=_mat_from_f(mats[1]), b2=_mat_from_f(mats[2]),
                    tgid=_mat_from_f(mats[3]))

    def box(self) -> np.ndarray:
        """B0 alone (columns are box vectors)."""
        m = np.zeros(9)
        check(self._L.moldy_gpu_get_state(self._h, *([None] * 9), _dp(m), None, None, None))
        return _mat_from_f(m)

    def forces(self) -> np.ndarray:
        f = [np.zeros(self.nm) for _ in range(3)]
        check(self._L.moldy_gpu_get_forces(self._h, *[_dp(a) for a in f]))
        return np.stack(f, axis=1)

    def density(self) -> dict:
        d = [np.zeros(self.nm) for _ in range(3)]
        check(self._L.moldy_gpu_get_density(self._h, *[_dp(a) for a in d]))
        return dict(rho=d[0], afrho=d[1], dafrho=d[2])

    def atomstress(self) -> np.ndarray:
        d = [np.zeros(self.nm) for _ in range(3)]
        check(self._L.moldy_gpu_get_atomstress(self._h, *[_dp(a) for a in d]))
        return np.stack(d, axis=1)

    def set_ntc(self, ntc: int):
        check(self._L.moldy_gpu_set_ntc(self._h, int(ntc)))

    # ------------------------------------------------ link cells / nlist
    def linkup(self):
        check(self._L.moldy_gpu_linkup(self._h))

    def relink(self):
        check(self._L.moldy_gpu_relink(self._h))

    def linkcells(self, ncell: int):
        l0 = np.zeros(ncell, dtype=np.int32)
        link = np.zeros(self.nm, dtype=np.int32)
        ic = np.zeros(self.nm, dtype=np.int32)
        check(self._L.moldy_gpu_get_linkcells(self._h, _ip(l0), _ip(link), _ip(ic)))
        return l0, link, ic

    def update_neighbourlist(self):
        check(self._L.moldy_gpu_update_neighbourlist(self._h))

    def neighbour_list(self):
        """(nlist[nm, nnbrs] 1-based, numn[nm]) -- Fortran NLIST(nnbrs, nm) memory."""
        nl = np.zeros(self.nm * self.nnbrs, dtype=np.int32)
        nn = np.zeros(self.nm, dtype=np.int32)
        check(self._L.moldy_gpu_get_neighbourlist(self._h, _ip(nl), _ip(nn)))
        return nl.reshape(self.nm, self.nnbrs), nn

    def reverse_list(self):
        """(rlist[nm, nnbrs] 1-based, numr[nm]): row i holds the atoms j whose
        neighbour-list rows hold i, i's own link cell first, then the mirror
        half stencil, each cell in chain order."""
        nl = np.zeros(self.nm * self.nnbrs, dtype=np.int32)
        nn = np.zeros(self.nm, dtype=np.int32)
        check(self._L.moldy_gpu_get_reverse_list(self._h, _ip(nl), _ip(nn)))
        return nl.reshape(self.nm, self.nnbrs), nn

    # ------------------------------------------------------------ hot path
    @staticmethod
    def _force_dict(o: _lib.ForceOut) -> dict:
        out = {"pe": o.pe, "vol": o.vol, "ntc": o.ntc, "rebuilt": bool(o.rebuilt)}
        for k in ("tp", "tk", "tc", "tg", "tgdot", "tgid", "fb"):
            out[k] = _mat_from_f(np.array(getattr(o, k)[:]))
        return out

    def force(self) -> dict:
        o = _lib.ForceOut()
        check(self._L.moldy_gpu_force(self._h, ctypes.byref(o)))
        return self._force_dict(o)

    def energy_forces_stress(self, out: dict | None = None):
        """(pe, real forces [nm,3], sigma [3,3]) as write_energy_forces_stress
        prints them (src/dynamics_m.F90:588-619) after a force evaluation:
        F = B0 f and sigma(i,j) = -sum_k b0(j,k) tp(i,k) / vol."""
        if out is None:
            out = self.force()
        b0 = self.box()
        f = self.forces() @ b0.T
        sigma = -(out["tp"] @ b0.T) / out["vol"]
        return out["pe"], f, sigma

    # --------------------------------------------------------------- adjoint
    @staticmethod
    def _grad_inputs(nm, g_force, g_stress):
        gf = None if g_force is None else _f64(np.asarray(g_force, dtype=np.float64).reshape(nm, 3).T)
        gs = _mat_f(g_stress)
        return gf, gs

    def table_gradients(self, g_energy=0.0, g_force=None, g_stress=None) -> dict:
        """dL/d(table node) for dL/dE = g_energy, dL/dF = g_force [nm,3] (real
        forces) and dL/dsigma = g_stress [3,3], at the last force evaluation."""
        gf, gs = self._grad_inputs(self.nm, g_force, g_stress)
        n = self.nlookup + 1
        t = [np.zeros(n) for _ in range(6)]
        check(self._L.moldy_gpu_table_gradients(self._h, float(g_energy), _dp(gf), _dp(gs),
                                                *[_dp(a) for a in t]))
        return dict(zip(["vee", "dvee", "phi", "dphi", "emb", "demb"], t))

    def knot_gradients(self, g_energy=0.0, g_force=None, g_stress=None) -> dict:
        """dL/d(av, rv, ap, rp) of the Fe-Fe knots set by set_up_fetm."""
        gf, gs = self._grad_inputs(self.nm, g_force, g_stress)
        nv, npk = self.n_knots
        out = [np.zeros(nv), np.zeros(nv), np.zeros(npk), np.zeros(npk)]
        check(self._L.moldy_gpu_knot_gradients(self._h, float(g_energy), _dp(gf), _dp(gs),
                                               *[_dp(a) for a in out]))
        return dict(zip(["av", "rv", "ap", "rp"], out))

    def velocityverlet(self) -> dict:
        o = _lib.ForceOut()
        check(self._L.moldy_gpu_velocityverlet(self._h, ctypes.byref(o)))
        return self._force_dict(o)

    def update_therm_avs(self) -> np.ndarray:
        s = np.zeros(3)
        check(self._L.moldy_gpu_update_therm_avs(self._h, _dp(s)))
        return s

    def md_init(self) -> dict:
        o = _lib.ForceOut()
        check(self._L.moldy_gpu_md_init(self._h, ctypes.byref(o)))
        return self._force_dict(o)

    def md_steps(self, nsteps: int, *, thermo: bool = True):
        """Runs nsteps mdloop iterations; returns a list of per-step thermo dicts."""
        if not thermo:
            check(self._L.moldy_gpu_md_steps(self._h, int(nsteps), None))
            return None
        arr = (_lib.Thermo * max(int(nsteps), 1))()
        check(self._L.moldy_gpu_md_steps(self._h, int(nsteps), arr))
        keys = [f[0] for f in _lib.Thermo._fields_]
        return [{k: getattr(arr[i], k) for k in keys} for i in range(int(nsteps))]

    def set_thermostat(self, nose: float, rqke: float):
        """simparam%nose and simparam%rqke of scalev; nose = 0 switches it off."""
        check(self._L.moldy_gpu_set_thermostat(self._h, float(nose), float(rqke)))

    def thermostat(self) -> dict:
        v = np.zeros(4)
        check(self._L.moldy_gpu_get_thermostat(self._h, _dp(v)))
        return {"nose": v[0], "rqke": v[1], "snhv": v[2], "thermotimer": v[3]}

    def scalev(self):
        check(self._L.moldy_gpu_scalev(self._h))

    def strainloops(self, loops: int, nsteps: int, *, temprq: float, tempsp: float = 0.0, nose: float = 0.0,
                    strx=None, thermo: bool = True):
        """The strain-loop driver of moldin (src/moldin.F90:417-437): each loop
        applies strx to B0 (when ivol != 0, keeping the old B0 in B2), raises
        the required temperature by tempsp, sets rqke = 1.5 bk temprq (nm - 3),
        then runs nsteps mdloop iterations with scalev (nose > 0).  Returns the
        per-step thermodynamics (if asked) and the final temprq."""
        from . import units
        records = []
        for _ in range(int(loops)):
            if strx is not None and self.params.ivol != 0:
                st = self.get_state()
                b0 = np.asarray(strx, dtype=np.float64) @ st["b0"]
                self.set_state(b0=b0, b2=st["b0"])
            temprq = temprq + tempsp
            rqke = 1.5 * units.BK * temprq * (self.nm - 3)
            self.set_thermostat(nose, rqke)
            r = self.md_steps(nsteps, thermo=thermo)
            if thermo:
                for rec in r:
                    rec["temprq"] = temprq
                records.extend(r)
        return records, temprq

    def energy_calc(self) -> np.ndarray:
        e = np.zeros(self.nm)
        check(self._L.moldy_gpu_energy_calc(self._h, _dp(e)))
        return e

    def synchronize(self):
        check(self._L.moldy_gpu_synchronize(self._h))

    # ------------------------------------------------------- instrumentation
    def stream_handle(self) -> int:
        """cudaStream_t (as an int) that all of this system's work runs on."""
        v = ctypes.c_void_p()
        check(self._L.moldy_gpu_get_stream(self._h, ctypes.byref(v)))
        return int(v.value or 0)

    def set_profiling(self, on: bool):
        check(self._L.moldy_gpu_set_profiling(self._h, int(bool(on))))

    def reset_kernel_stats(self):
        check(self._L.moldy_gpu_reset_kernel_stats(self._h))

    def autotune(self, nreps: int = 5) -> dict:
        """Times each compiled variant of the screening-density and force
        passes on the current configuration and keeps the fastest."""
        import numpy as _np
        t = _np.zeros(3 * _lib.TUNE_VARIANTS)
        ch = _np.zeros(3, dtype=_np.int32)
        check(self._L.moldy_gpu_autotune(self._h, int(nreps), _dp(t), _ip(ch)))
        nv = _lib.TUNE_VARIANTS
        return {"chosen": {"screen_density": int(ch[0]), "forces": int(ch[2])},
                "ms": {"screen_density": t[0:nv].tolist(), "forces": t[2 * nv:3 * nv].tolist()}}

    def list_stats(self) -> dict:
        """Directed interacting pairs of the last force evaluation, the number
        of intermediate-list builds so far and the list entries the screening
        pass reads per step."""
        v = np.zeros(3)
        check(self._L.moldy_gpu_get_list_stats(self._h, _dp(v)))
        return {"pairs": float(v[0]), "mid_builds": int(v[1]), "screened": float(v[2])}

    def pair_count(self) -> float:
        return self.list_stats()["pairs"]

    def set_mid_skin(self, skin: float):
        """Skin (A) of the intermediate list; a tuning knob, results unchanged."""
        check(self._L.moldy_gpu_set_mid_skin(self._h, float(skin)))

    def set_outer_skin(self, skin: float):
        """Skin (A) of the outer list the intermediate list is filtered from;
        a tuning knob, results unchanged."""
        check(self._L.moldy_gpu_set_outer_skin(self._h, float(skin)))

    def outer_builds(self) -> int:
        n = ctypes.c_int32(0)
        check(self._L.moldy_gpu_get_outer_builds(self._h, ctypes.byref(n)))
        return int(n.value)

    def set_variants(self, screen: int, density: int, forces: int):
        check(self._L.moldy_gpu_set_variants(self._h, int(screen), int(density), int(forces)))

    def kernel_stats(self) -> dict:
        """{family: (total_ms, launches)} since the last reset."""
        out = {}
        for k in range(_lib.KERNEL_FAMILIES):
            ms = ctypes.c_double()
            n = ctypes.c_int64()
            check(self._L.moldy_gpu_kernel_stats(self._h, k, ctypes.byref(ms), ctypes.byref(n)))
            out[self._L.moldy_gpu_kernel_name(k).decode()] = (ms.value, int(n.value))
        return out
