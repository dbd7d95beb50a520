"""Many independent supercells on one GPU (the ``moldy_gpu_batch_*`` C ABI).

Each system's energy, forces and virial are those of force() + energy_calc()
(src/dynamics_m.F90:135-483) in lookup mode, and :meth:`MoldyBatch.quench` is
quench_m::quench with VA14CD and derivs (src/quench_m.F90:100-551) at a fixed
box, run for every system at once on the device.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check
from .system import _dp, _f64, _mat_f, _mat_from_f


class MoldyBatch:
    """nsys systems of natoms[s] atoms each, concatenated in system order."""

    def __init__(self, natoms, *, press=0.0, device=0):
        self._L = _lib.load()
        na = np.ascontiguousarray(natoms, dtype=np.int32)
        h = _lib.H()
        check(self._L.moldy_gpu_batch_create(len(na), na.ctypes.data_as(_lib.I), float(press), int(device),
                                             ctypes.byref(h)))
        self._h = h
        self.natoms = na.astype(np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)])
        self.nsys = len(na)
        self.ntot = int(self.offsets[-1])

    @classmethod
    def from_workloads(cls, ws, *, nlookup=5000, device=0):
        b = cls([w.nm for w in ws], press=ws[0].press, device=device)
        b.set_up_fetm(ws[0].coeffs, nlookup=nlookup)
        b.set_state(np.concatenate([w.x0 for w in ws]), [w.b0 for w in ws],
                    np.concatenate([w.atomic_mass for w in ws]))
        return b

    def close(self):
        if getattr(self, "_h", None):
            self._L.moldy_gpu_batch_destroy(self._h)
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

    def set_up_fetm(self, coeffs, *, nlookup=5000):
        av, rv, ap, rp = (_f64(v) for v in (coeffs.av, coeffs.rv, coeffs.ap, coeffs.rp))
        check(self._L.moldy_gpu_batch_set_fetm_fe(self._h, len(av), _dp(av), _dp(rv), len(ap), _dp(ap), _dp(rp),
                                                  int(nlookup)))
        self.nlookup = int(nlookup)

    def set_state(self, x0=None, b0=None, mass=None):
        """x0: (ntot, 3) fractional positions; b0: nsys 3x3 boxes (columns are
        box vectors); mass: (ntot,)."""
        cols = [None, None, None]
        if x0 is not None:
            a = np.asarray(x0, dtype=np.float64).reshape(self.ntot, 3)
            cols = [_f64(a[:, k]) for k in range(3)]
        bb = None
        if b0 is not None:
            bb = _f64(np.concatenate([_mat_f(m) for m in b0]))
        m = None if mass is None else _f64(mass)
        check(self._L.moldy_gpu_batch_set_state(self._h, *[_dp(c) for c in cols], _dp(bb), _dp(m)))

    def set_positions(self, xyz):
        """(ntot, 3) C-contiguous float64 fractional positions in one copy
        (pinned host memory copies fastest)."""
        a = self._xyz(xyz)
        check(self._L.moldy_gpu_batch_set_positions(self._h, _dp(a)))

    def forces_xyz_into(self, out):
        """Fractional forces into a preallocated (ntot, 3) C-contiguous float64 array."""
        check(self._L.moldy_gpu_batch_get_forces_xyz(self._h, _dp(self._xyz(out))))

    def _xyz(self, a):
        if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous \
                or a.shape != (self.ntot, 3):
            raise ValueError("needs a C-contiguous float64 array of shape (ntot, 3)")
        return a

    def get_state(self) -> np.ndarray:
        c = [np.zeros(self.ntot) for _ in range(3)]
        check(self._L.moldy_gpu_batch_get_state(self._h, *[_dp(a) for a in c]))
        return np.stack(c, axis=1)

    def force(self) -> dict:
        """One evaluation of every system: per-system arrays pe_calc
        (energy_calc), pe (force routine), fmax (largest |B0 f|), vol, tp."""
        o = np.zeros(13 * self.nsys)
        check(self._L.moldy_gpu_batch_force(self._h, _dp(o)))
        o = o.reshape(self.nsys, 13)
        return {"pe_calc": o[:, 0].copy(), "pe": o[:, 1].copy(), "fmax": o[:, 2].copy(), "vol": o[:, 3].copy(),
                "tp": np.stack([_mat_from_f(o[s, 4:13]) for s in range(self.nsys)])}

    def force_into(self, out):
        """One evaluation of every system with its per-system results written
        raw into a preallocated contiguous float64 array of 13 * nsys: pe_calc,
        pe, fmax, vol and tp (column-major 3x3) per system."""
        if not isinstance(out, np.ndarray) or out.dtype != np.float64 or not out.flags.c_contiguous \
                or out.size != 13 * self.nsys:
            raise ValueError("needs a contiguous float64 array of 13 * nsys")
        check(self._L.moldy_gpu_batch_force(self._h, _dp(out)))

    def forces(self) -> np.ndarray:
        c = [np.zeros(self.ntot) for _ in range(3)]
        check(self._L.moldy_gpu_batch_get_forces(self._h, *[_dp(a) for a in c]))
        return np.stack(c, axis=1)

    def forces_into(self, fx, fy, fz):
        """Fractional forces into three preallocated contiguous float64 arrays."""
        for a in (fx, fy, fz):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != (self.ntot,):
                raise ValueError("forces_into needs contiguous float64 arrays of length ntot")
        check(self._L.moldy_gpu_batch_get_forces(self._h, _dp(fx), _dp(fy), _dp(fz)))

    def energies(self):
        a, b = np.zeros(self.ntot), np.zeros(self.ntot)
        check(self._L.moldy_gpu_batch_get_energies(self._h, _dp(a), _dp(b)))
        return a, b

    def density(self) -> dict:
        d = [np.zeros(self.ntot) for _ in range(3)]
        check(self._L.moldy_gpu_batch_get_density(self._h, *[_dp(a) for a in d]))
        return dict(rho=d[0], afrho=d[1], dafrho=d[2])

    def quench(self, maxfn=1000, criterion=0, fmax=1e-4) -> dict:
        """VA14CD quench of every system; criterion 0 is the reference's
        (sum of squared gradient <= 5e-7 nm), 1 is max |B0 f| <= fmax."""
        o = np.zeros(8 * self.nsys)
        check(self._L.moldy_gpu_batch_quench(self._h, int(maxfn), int(criterion), float(fmax), _dp(o)))
        o = o.reshape(self.nsys, 8)
        return {"f": o[:, 0].copy(), "pe": o[:, 1].copy(), "gsumsq": o[:, 2].copy(), "fmax": o[:, 3].copy(),
                "nfev": o[:, 4].astype(np.int64), "iterations": o[:, 5].astype(np.int64),
                "iflag": o[:, 6].astype(np.int64)}

    def set_tiles(self, lanes=8, staged=256):
        check(self._L.moldy_gpu_batch_set_tiles(self._h, int(lanes), int(staged)))

    def set_precision(self, precision="fp64"):
        """"fp64" or "mixed" (FP32 separations, tables and pair forces, FP64
        sums) for the density and force passes of :meth:`force`.  The quench
        always evaluates in FP64, as its line search needs."""
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision is 'fp64' or 'mixed'")
        check(self._L.moldy_gpu_batch_set_precision(self._h, 1 if precision == "mixed" else 0))

    def autotune(self, nreps: int = 3) -> dict:
        """Chooses the tile lanes per home atom, the gather width and, where
        the persistent evaluation applies, its lanes per atom on the live
        configuration (moldy_gpu_batch_autotune); returns the mean evaluation
        times (ms) and the choice (atom_lanes 0: not tuned)."""
        t = np.zeros(10)
        ch = (ctypes.c_int32 * 3)()
        check(self._L.moldy_gpu_batch_autotune(self._h, int(nreps), _dp(t), ch))
        out = {"lanes_ms": dict(zip((4, 8, 16, 32), t[:4].tolist())),
               "gather_ms": dict(zip((1, 2, 4), t[4:7].tolist())),
               "chosen": {"lanes": int(ch[0]), "gather": int(ch[1]), "atom_lanes": int(ch[2])}}
        if ch[2]:
            out["atom_lanes_ms"] = dict(zip((1, 2, 4), t[7:].tolist()))
        return out

    def set_persistent(self, enable: bool = True):
        """Whether :meth:`force` may evaluate every system in one persistent
        launch (mixed precision, energy_calc off, every atom heavier than 0.05)."""
        check(self._L.moldy_gpu_batch_set_persistent(self._h, 1 if enable else 0))

    def set_atom_lanes(self, lanes: int):
        """Lanes per atom (1, 2, 4) of the persistent evaluation's passes."""
        check(self._L.moldy_gpu_batch_set_atom_lanes(self._h, int(lanes)))

    def persistent_applies(self) -> bool:
        """True when :meth:`force` runs the persistent evaluation."""
        v = ctypes.c_int32(0)
        check(self._L.moldy_gpu_batch_persistent_applies(self._h, ctypes.byref(v)))
        return bool(v.value)

    def eval_times(self) -> dict:
        """Device times (ms) of the persistent evaluation with every list
        current and with every list rebuilt in the same launch."""
        t = np.zeros(2)
        check(self._L.moldy_gpu_batch_eval_times(self._h, _dp(t)))
        return {"current": float(t[0]), "rebuilt": float(t[1])}

    def set_references(self, f_ref, sigma_ref):
        """Reference real forces (one (nm_s, 3) array per system, or one (ntot, 3)
        array in atom order) and stresses ((nsys, 3, 3), sigma(i,j) =
        -sum_k b0(j,k) tp(i,k) / vol, model units) for :meth:`force_matching`."""
        f = np.ascontiguousarray(np.concatenate(f_ref) if isinstance(f_ref, (list, tuple)) else f_ref,
                                 dtype=np.float64).reshape(self.ntot, 3)
        sg = np.asarray(sigma_ref, dtype=np.float64).reshape(self.nsys, 3, 3)
        sref = np.ascontiguousarray(np.stack([m.ravel(order="F") for m in sg]))
        check(self._L.moldy_gpu_batch_set_references(self._h, _dp(f), _dp(sref)))

    def force_matching(self, w_force=1.0, w_stress=1.0):
        """One FP64 evaluation of every system: the per-system force-matching
        loss against the references and dL/d(table) of their sum (dict of the
        six tables; vee and emb get none)."""
        loss = np.zeros(self.nsys)
        nb = self.nlookup + 1
        g = np.zeros(6 * nb)
        check(self._L.moldy_gpu_batch_force_matching(self._h, float(w_force), float(w_stress), _dp(loss), _dp(g)))
        names = ("vee", "dvee", "phi", "dphi", "emb", "demb")
        return loss, {k: g[i * nb:(i + 1) * nb].copy() for i, k in enumerate(names)}

    def kernel_times(self, rebuild=False) -> dict:
        """One evaluation with its four launches timed (ms): the list check,
        the tile screen, the density pass and the force pass."""
        t = np.zeros(4)
        check(self._L.moldy_gpu_batch_kernel_times(self._h, 1 if rebuild else 0, _dp(t)))
        return dict(zip(("prepare", "tile_screen", "density", "forces"), t.tolist()))

    def set_energy_calc(self, enable=True):
        """Whether force() also forms energy_calc's per-atom energies (the
        exact pair function; default on).  The quench always forms them."""
        check(self._L.moldy_gpu_batch_set_energy_calc(self._h, 1 if enable else 0))

    def set_gather(self, entries=4):
        """Row entries a thread gathers at a time in the per-atom passes (1, 2, 4)."""
        check(self._L.moldy_gpu_batch_set_gather(self._h, int(entries)))

    def set_skin(self, skin=0.3):
        """Verlet skin of the per-system lists (A); 0 rebuilds whenever an atom moved."""
        check(self._L.moldy_gpu_batch_set_skin(self._h, float(skin)))

    def list_stats(self) -> dict:
        """System list builds and system evaluations since creation."""
        v = (ctypes.c_int64 * 2)()
        check(self._L.moldy_gpu_batch_list_stats(self._h, v))
        return {"builds": int(v[0]), "evaluations": int(v[1])}

    def row_entries(self) -> int:
        """Compact-row entries summed over all atoms (pairs within the list
        radius, both directions), as the last evaluation left them."""
        v = ctypes.c_int64(0)
        check(self._L.moldy_gpu_batch_row_entries(self._h, ctypes.byref(v)))
        return int(v.value)

    def launches(self) -> int:
        v = ctypes.c_int64(0)
        check(self._L.moldy_gpu_batch_launches(self._h, ctypes.byref(v)))
        return int(v.value)

    def stream_handle(self) -> int:
        p = ctypes.c_void_p()
        check(self._L.moldy_gpu_batch_get_stream(self._h, ctypes.byref(p)))
        return int(p.value or 0)

    def split(self, arr):
        """Per-system views of a concatenated per-atom array."""
        return [arr[self.offsets[s]:self.offsets[s + 1]] for s in range(self.nsys)]


def gather_system_results(local: dict, assignment, nsys: int, group=None) -> dict:
    """Per-system results of a batch sharded over ranks, on every rank.

    ``local`` maps names to this rank's arrays, first dimension = its
    systems in the order of ``assignment[rank]`` (``adjoint.shard_configs``
    gives such an assignment); ``assignment[r]`` lists the global indices of
    rank r's systems.  One all_gather of a packed float64 tensor per rank
    (padded to the largest shard; on the GPU under NCCL, on the host under
    gloo) places every system's row at its global index.  Without an
    initialised process group the local arrays are the whole batch."""
    import torch
    import torch.distributed as dist
    names = sorted(local)
    if not (dist.is_available() and dist.is_initialized()):
        return {k: np.asarray(local[k]) for k in names}
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = list(assignment[rank])
    arrs = [np.asarray(local[k], dtype=np.float64).reshape(len(mine), -1) for k in names]
    widths = [a.shape[1] for a in arrs]
    width = int(sum(widths))
    rows = max(len(a) for a in assignment)
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    buf = torch.zeros((rows, width), dtype=torch.float64, device=device)
    if mine:
        buf[:len(mine)] = torch.from_numpy(np.concatenate(arrs, axis=1)).to(device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = {}
    off = 0
    for k, wdt, a in zip(names, widths, arrs):
        full = np.zeros((nsys, wdt))
        for r in range(world):
            p = parts[r].cpu().numpy()
            for i, sidx in enumerate(assignment[r]):
                full[sidx] = p[i, off:off + wdt]
        shape = np.asarray(local[k]).shape[1:]
        out[k] = full.reshape((nsys,) + tuple(shape))
        off += wdt
    return out
