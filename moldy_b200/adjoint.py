"""Force-matching gradients: torch.autograd.Function wrappers over the C ABI.

The forward of each Function is one force evaluation on the GPU
(``moldy_gpu_force``) and returns, for one configuration, the energy, the real
forces and the stress that the reference prints in ``efs.out``
(``write_energy_forces_stress``, src/dynamics_m.F90:588-619):

    E = pe,   F = B0 f  [nm, 3],   sigma(i,j) = -sum_k b0(j,k) tp(i,k) / vol.

The backward calls the hand-written adjoint kernels
(``moldy_gpu_table_gradients`` / ``moldy_gpu_knot_gradients``), which
recompute rho on the device and scatter dL/d(table) through shared-memory
histograms.  Parameters are either the six lookup tables (``EAMTables``) or
the Fe-Fe knot parameters av, rv, ap, rp of src/fetransmetal.F90:74-77
(``EAMKnots``); F(rho) = -sqrt(rho) has no parameters.

Tensors are float64 on the host; the state of each configuration lives in a
:class:`MoldySystem`.  A backward whose system has been re-evaluated since its
forward re-runs that forward first, so one system can serve many
configurations.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import check
from .potentials import FeFeCoefficients
from .system import MoldySystem, _dp, _f64

TABLE_NAMES = ("vee", "dvee", "phi", "dphi", "emb", "demb")
KNOT_NAMES = ("av", "rv", "ap", "rp")


def _t(a) -> torch.Tensor:
    return torch.as_tensor(np.asarray(a, dtype=np.float64))


def _np_grad(g):
    return None if g is None else g.detach().to(torch.float64).cpu().numpy()


def _evaluate(system: MoldySystem):
    """One force evaluation with fresh link cells and neighbour list."""
    system.linkup()
    system.set_ntc(0)
    e, f, s = system.energy_forces_stress()
    system._adj_generation = getattr(system, "_adj_generation", 0) + 1
    return e, f, s, system._adj_generation


class _Saved:
    """State a backward needs to re-create its forward on a shared system."""

    def __init__(self, system: MoldySystem, generation: int, setter):
        self.system = system
        self.generation = generation
        st = system.get_state()
        self.x0, self.b0 = st["x0"], st["b0"]
        self.setter = setter

    def restore(self):
        s = self.system
        if getattr(s, "_adj_generation", 0) == self.generation:
            return
        self.setter()
        s.set_state(x0=self.x0, b0=self.b0)
        _evaluate(s)


class EAMTables(torch.autograd.Function):
    """(E, F, sigma) of one configuration as functions of the six tables.

    ``apply(system, ranges, vee, dvee, phi, dphi, emb, demb)`` with ranges =
    (rmin, rmax, rhomin, rhomax) and tables of nlookup+1 float64 values."""

    @staticmethod
    def forward(ctx, system, ranges, vee, dvee, phi, dphi, emb, demb):
        tabs = {k: _f64(t.detach().cpu().numpy()) for k, t in zip(TABLE_NAMES, (vee, dvee, phi, dphi, emb, demb))}
        rmin, rmax, rhomin, rhomax = (float(v) for v in ranges)

        def setter():
            system.set_tables(tabs, rmin=rmin, rmax=rmax, rhomin=rhomin, rhomax=rhomax)

        setter()
        e, f, s, gen = _evaluate(system)
        ctx.saved = _Saved(system, gen, setter)
        return _t(e), _t(f), _t(s)

    @staticmethod
    def backward(ctx, g_e, g_f, g_s):
        sv = ctx.saved
        sv.restore()
        g = sv.system.table_gradients(0.0 if g_e is None else float(g_e), _np_grad(g_f), _np_grad(g_s))
        return (None, None) + tuple(_t(g[k]) for k in TABLE_NAMES)


class EAMKnots(torch.autograd.Function):
    """(E, F, sigma) of one configuration as functions of the Fe-Fe knots.

    ``apply(system, nlookup, av, rv, ap, rp)``; lookup mode with nlookup
    intervals, as potential_set_lookup builds the tables."""

    @staticmethod
    def forward(ctx, system, nlookup, av, rv, ap, rp):
        coeffs = FeFeCoefficients(*(_f64(t.detach().cpu().numpy()) for t in (av, rv, ap, rp)))

        def setter():
            system.set_up_fetm(coeffs, uselookup=True, nlookup=int(nlookup))

        setter()
        e, f, s, gen = _evaluate(system)
        ctx.saved = _Saved(system, gen, setter)
        return _t(e), _t(f), _t(s)

    @staticmethod
    def backward(ctx, g_e, g_f, g_s):
        sv = ctx.saved
        sv.restore()
        g = sv.system.knot_gradients(0.0 if g_e is None else float(g_e), _np_grad(g_f), _np_grad(g_s))
        return (None, None) + tuple(_t(g[k]) for k in KNOT_NAMES)


def _force_matching_share(system, coeffs, nlookup, configs, refs, w_force, w_stress):
    """Loss and summed table gradients of some configurations on one system."""
    system.set_up_fetm(coeffs, uselookup=True, nlookup=int(nlookup))
    loss = 0.0
    acc = {k: np.zeros(int(nlookup) + 1) for k in TABLE_NAMES}
    for (x0, b0), (f_ref, s_ref) in zip(configs, refs):
        system.set_state(x0=x0, b0=b0)
        _, f, sig, _ = _evaluate(system)
        df = f - np.asarray(f_ref, dtype=np.float64)
        ds = sig - np.asarray(s_ref, dtype=np.float64)
        loss += w_force * float((df * df).sum()) + w_stress * float((ds * ds).sum())
        g = system.table_gradients(0.0, 2.0 * w_force * df, 2.0 * w_stress * ds)
        for k in TABLE_NAMES:
            acc[k] += g[k]
    return loss, acc


class ForceMatchingKnots(torch.autograd.Function):
    """The force-matching loss of many configurations,
    sum_c w_force |F_c - F_c^ref|^2 + w_stress |sigma_c - sigma_c^ref|^2, as a
    function of the Fe-Fe knots.  The loss is a scalar, so its gradient is
    formed in the forward pass: the tables are built once per system, each
    configuration is evaluated once and its table gradients summed, and one
    contraction with d(table)/d(knot) gives dL/d(knot); backward scales it.

    ``apply(systems, configs, refs, w_force, w_stress, nlookup, av, rv, ap,
    rp)``; systems is one MoldySystem or a list of them (each on its own CUDA
    stream): with k systems, host threads evaluate configuration c on system
    c mod k, so their launches and copies overlap, and the shares are summed
    in system order.  configs[c] = (x0 [nm,3] fractional, b0 3x3), refs[c] =
    (F_ref [nm,3] real forces, sigma_ref 3x3)."""

    @staticmethod
    def forward(ctx, systems, configs, refs, w_force, w_stress, nlookup, av, rv, ap, rp):
        coeffs = FeFeCoefficients(*(_f64(t.detach().cpu().numpy()) for t in (av, rv, ap, rp)))
        systems = list(systems) if isinstance(systems, (list, tuple)) else [systems]
        k = len(systems)
        shares = [(systems[t], coeffs, nlookup, configs[t::k], refs[t::k], w_force, w_stress) for t in range(k)]
        if k == 1:
            results = [_force_matching_share(*shares[0])]
        else:
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(max_workers=k) as pool:
                results = list(pool.map(lambda a: _force_matching_share(*a), shares))
        loss = 0.0
        acc = {name: np.zeros(int(nlookup) + 1) for name in TABLE_NAMES}
        for l, g in results:
            loss += l
            for name in TABLE_NAMES:
                acc[name] += g[name]
        kg = fetm_knot_vjp(coeffs, acc, int(nlookup))
        ctx.grads = [torch.as_tensor(kg[name]) for name in KNOT_NAMES]
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        return (None,) * 6 + tuple(g * t for t in ctx.grads)


class BatchForceMatchingKnots(torch.autograd.Function):
    """The force-matching loss of every configuration held by a
    :class:`moldy_b200.MoldyBatch` (its references set with
    ``set_references``), as a function of the Fe-Fe knots.  The forward builds
    the tables from the knots, runs one FP64 evaluation of all systems, forms
    the loss and the table gradients on the device (moldy_gpu_batch_force_matching)
    and contracts them with d(table)/d(knot) on the host; backward scales the
    stored gradient.  ``apply(batch, w_force, w_stress, nlookup, av, rv, ap, rp)``."""

    @staticmethod
    def forward(ctx, batch, w_force, w_stress, nlookup, av, rv, ap, rp):
        coeffs = FeFeCoefficients(*(_f64(t.detach().cpu().numpy()) for t in (av, rv, ap, rp)))
        batch.set_up_fetm(coeffs, nlookup=int(nlookup))
        loss, tg = batch.force_matching(w_force, w_stress)
        kg = fetm_knot_vjp(coeffs, tg, int(nlookup))
        ctx.grads = [torch.as_tensor(kg[name]) for name in KNOT_NAMES]
        ctx.loss_per_system = loss
        return torch.tensor(float(loss.sum()), dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        return (None,) * 4 + tuple(g * t for t in ctx.grads)


def batch_force_matching_knots(batch, knots: dict, *, w_force=1.0, w_stress=1.0, nlookup: int = 5000):
    """Scalar force-matching loss of every configuration of a MoldyBatch,
    differentiable in the knots dict {av, rv, ap, rp} of torch tensors
    (BatchForceMatchingKnots)."""
    return BatchForceMatchingKnots.apply(batch, float(w_force), float(w_stress), int(nlookup),
                                         *[knots[k] for k in KNOT_NAMES])


def force_matching_knots(systems, configs, refs, knots: dict, *, w_force=1.0, w_stress=1.0, nlookup: int = 5000):
    """Scalar force-matching loss of many configurations on one system or a
    list of systems, differentiable in the knots dict {av, rv, ap, rp} of
    torch tensors (ForceMatchingKnots)."""
    return ForceMatchingKnots.apply(systems, configs, refs, float(w_force), float(w_stress), int(nlookup),
                                    *[knots[k] for k in KNOT_NAMES])


def eam_tables(system, tables: dict, ranges=(0.0, 6.0, 0.0, 10000.0)):
    """(E, F, sigma) differentiable in the tables dict of torch tensors."""
    return EAMTables.apply(system, tuple(ranges), *[tables[k] for k in TABLE_NAMES])


def eam_knots(system, knots: dict, nlookup: int = 5000):
    """(E, F, sigma) differentiable in the knots dict {av, rv, ap, rp} of torch tensors."""
    return EAMKnots.apply(system, int(nlookup), *[knots[k] for k in KNOT_NAMES])


def force_matching_loss(evaluate, systems, references, *, w_force=1.0, w_stress=1.0):
    """sum_c w_force |F_c - F_c^ref|^2 + w_stress |sigma_c - sigma_c^ref|^2.

    evaluate(system) -> (E, F, sigma) differentiable in the parameters;
    references[c] = (F_ref [nm,3], sigma_ref [3,3]) as arrays or tensors."""
    loss = torch.zeros((), dtype=torch.float64)
    for s, (f_ref, s_ref) in zip(systems, references):
        _, f, sig = evaluate(s)
        loss = loss + w_force * ((f - _t(f_ref)) ** 2).sum() + w_stress * ((sig - _t(s_ref)) ** 2).sum()
    return loss


# ------------------------------------------------------------ host helpers --
def fetm_tables(coeffs: FeFeCoefficients, nlookup: int = 5000) -> dict:
    """The six lookup tables of the Fe-Fe knots (host, no device needed)."""
    L = _lib.load()
    av, rv, ap, rp = (_f64(v) for v in (coeffs.av, coeffs.rv, coeffs.ap, coeffs.rp))
    t = [np.zeros(nlookup + 1) for _ in range(6)]
    check(L.moldy_fetm_build_tables(len(av), _dp(av), _dp(rv), len(ap), _dp(ap), _dp(rp), int(nlookup),
                                    *[_dp(a) for a in t]))
    return dict(zip(TABLE_NAMES, t))


def fetm_knot_vjp(coeffs: FeFeCoefficients, table_grads: dict, nlookup: int = 5000) -> dict:
    """Contracts dL/d(table) with d(table)/d(knot) (host, no device needed)."""
    L = _lib.load()
    av, rv, ap, rp = (_f64(v) for v in (coeffs.av, coeffs.rv, coeffs.ap, coeffs.rp))
    g = [None if table_grads.get(k) is None else _f64(table_grads[k]) for k in TABLE_NAMES]
    out = [np.zeros(len(av)), np.zeros(len(av)), np.zeros(len(ap)), np.zeros(len(ap))]
    check(L.moldy_fetm_knot_vjp(len(av), _dp(av), _dp(rv), len(ap), _dp(ap), _dp(rp), int(nlookup),
                                *[_dp(a) for a in g], *[_dp(a) for a in out]))
    return dict(zip(KNOT_NAMES, out))


# --------------------------------------------------------- sharding (N>1) --
def shard_configs(natoms, world_size: int) -> list:
    """Greedy atom-count bin-pack of configurations onto ranks: largest first,
    each to the least-loaded rank (ties to the lowest rank).  Returns one list
    of configuration indices per rank, each in ascending order."""
    load = [0] * world_size
    out = [[] for _ in range(world_size)]
    for c in sorted(range(len(natoms)), key=lambda c: (-int(natoms[c]), c)):
        r = min(range(world_size), key=lambda k: (load[k], k))
        out[r].append(c)
        load[r] += int(natoms[c])
    return [sorted(v) for v in out]


def allreduce_gradients(grads, group=None):
    """Sums per-rank parameter gradients over all ranks (one all_reduce per
    tensor, in the order given, identical on every rank)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return grads
    for g in grads:
        dist.all_reduce(g, op=dist.ReduceOp.SUM, group=group)
    return grads
