"""GPU parity of the adjoint (dE/dtheta, dF/dtheta, dsigma/dtheta).

Three independent checks of the CUDA backward:
* the FP64 torch restatement of the forward (tests/eam_torch.py, pinned to
  the oracle on CPU) differentiated by torch autograd: table gradients within
  1e-9 norm-wise;
* central finite differences (h = 1e-6) of the GPU forward: table nodes and
  all sixteen knots within 1e-6 relative;
* central finite differences (h = 1e-6) of the oracle's FP64 forward for the
  knot gradients, within 1e-6 relative.
The loss is a fixed random linear functional L = gE E + sum gF.F + sum gS:sigma
(its gradient is exactly the vector-Jacobian product the adjoint computes),
and a force-matching loss through torch.autograd.Function.
"""
import numpy as np
import pytest
import torch

from moldy_b200 import FE_FE, FeFeCoefficients, MoldyError, MoldySystem
from moldy_b200 import adjoint as adj
from moldy_b200 import workloads as wl
from tests.eam_torch import NAMES, eam_forward, half_pairs, torch_tables
from tests.helpers import real_forces, rel_norm_err

pytestmark = pytest.mark.gpu


def fm_config(seed: int, n: int = 6, sigma: float = 0.12):
    rng = np.random.default_rng(seed)
    return wl.make_workload(n, sigma=sigma, temperature=0.0, ivol=1, seed=seed,
                            strain=wl.random_symmetric_strain(rng, 0.03))


def cotangents(nm, seed=9):
    rng = np.random.default_rng(seed)
    g_s = rng.normal(size=(3, 3))
    return 1.0, rng.normal(size=(nm, 3)), g_s + g_s.T


def linear_loss(e, f, s, ct):
    g_e, g_f, g_s = ct
    return g_e * e + float(np.sum(g_f * f)) + float(np.sum(g_s * s))


def gpu_eval(sys_, tables=None, coeffs=None):
    if tables is not None:
        sys_.set_tables(tables)
    if coeffs is not None:
        sys_.set_up_fetm(coeffs, uselookup=True, nlookup=5000)
    sys_.linkup()
    sys_.set_ntc(0)
    return sys_.energy_forces_stress()


@pytest.fixture(scope="module")
def case(gpu_lib, oracle_mod):
    w = fm_config(3)
    s = MoldySystem.from_workload(w, uselookup=True)
    e, f, sig = gpu_eval(s)
    o = oracle_mod.from_workload(w, uselookup=True, threads=4)
    o.force()
    yield dict(w=w, s=s, o=o, e=e, f=f, sig=sig, tabs=s.tables())
    s.close()


def test_forward_matches_torch_reference(case):
    w, o = case["w"], case["o"]
    i, j = half_pairs(*o.nlist())
    st = o.get_state()
    e, f, s = eam_forward(st["x0"], st["b0"], i, j, w.atomic_mass, torch_tables(case["tabs"], False))
    assert abs(case["e"] - e.item()) <= 1e-10 * abs(e.item())
    assert rel_norm_err(case["f"], f.numpy()) <= 1e-10
    assert rel_norm_err(case["sig"], s.numpy()) <= 1e-10


def test_table_gradients_match_autograd_reference(case):
    w, o, s = case["w"], case["o"], case["s"]
    ct = cotangents(w.nm)
    got = s.table_gradients(*ct)
    i, j = half_pairs(*o.nlist())
    st = o.get_state()
    tt = torch_tables(case["tabs"])
    e, f, sig = eam_forward(st["x0"], st["b0"], i, j, w.atomic_mass, tt)
    loss = ct[0] * e + (torch.as_tensor(ct[1]) * f).sum() + (torch.as_tensor(ct[2]) * sig).sum()
    loss.backward()
    for k in NAMES:
        ref = tt[k].grad.numpy()
        assert np.linalg.norm(ref) > 0.0, k
        assert rel_norm_err(got[k], ref) <= 1e-9, k


def test_table_gradients_finite_differences(case):
    """Central differences (h = 1e-6) of the GPU forward at nodes inside and
    beyond the table cut.  dvee and dphi do not enter E, so their nodes are
    checked on the force/stress part of the loss alone; the tolerance is 1e-6
    relative plus the rounding floor of the difference quotient."""
    w, s = case["w"], case["s"]
    ct_full = cotangents(w.nm)
    ct_fs = (0.0,) + ct_full[1:]
    got_full = s.table_gradients(*ct_full)
    got_fs = s.table_gradients(*ct_fs)
    tabs = case["tabs"]
    rho = s.density()["rho"]
    h = 1e-6
    r_nodes = [int(r / 6.0 * 5000) for r in (2.31, 2.52, 2.87, 3.3, 4.05, 5.2)]
    e_nodes = sorted({int(v / 10000.0 * 5000) for v in np.quantile(rho, [0.05, 0.5, 0.95])})
    checks = [(k, n) for k in ("vee", "dvee", "phi", "dphi") for n in r_nodes]
    checks += [(k, n) for k in ("emb", "demb") for n in e_nodes]
    try:
        for name, node in checks:
            ct, got = (ct_fs, got_fs) if name in ("dvee", "dphi") else (ct_full, got_full)
            vals = []
            for sgn in (1.0, -1.0):
                t = {k: v.copy() for k, v in tabs.items()}
                t[name][node] += sgn * h
                vals.append(linear_loss(*gpu_eval(s, tables=t), ct))
            fd = (vals[0] - vals[1]) / (2 * h)
            g = got[name][node]
            floor = 8 * np.finfo(np.float64).eps * abs(vals[0]) / (2 * h)
            assert abs(g) > 1e-3, (name, node, g)
            assert abs(fd - g) <= 1e-6 * abs(g) + floor, (name, node, fd, g, floor)
    finally:
        gpu_eval(s, tables=tabs)


def _shift(coeffs, name, k, h):
    d = {f: np.array(getattr(coeffs, f), dtype=np.float64) for f in ("av", "rv", "ap", "rp")}
    d[name][k] += h
    return FeFeCoefficients(**d)


def test_knot_gradients_finite_differences_gpu_and_oracle(case, oracle_mod):
    """dL/dknot against central differences of the GPU forward and of the
    oracle's FP64 forward (the reference gradient)."""
    w, s = case["w"], case["s"]
    ct = cotangents(w.nm)
    gpu_eval(s, coeffs=FE_FE)
    got = s.knot_gradients(*ct)
    h = 1e-6
    o = oracle_mod.from_workload(w, uselookup=True, threads=4)

    def oracle_loss(c):
        o.set_fetm(c.av, c.rv, c.ap, c.rp)
        o.set_lookup(True, 5000)
        o.ntc = 0
        o.force()
        fo = o.force_out()
        b0 = o.get_state()["b0"]
        return linear_loss(fo["pe"], real_forces(o.forces(), b0), -(fo["tp"] @ b0.T) / fo["vol"], ct)

    try:
        for name in adj.KNOT_NAMES:
            fd_gpu = np.zeros(len(got[name]))
            fd_orc = np.zeros(len(got[name]))
            for k in range(len(fd_gpu)):
                cp, cm = _shift(FE_FE, name, k, h), _shift(FE_FE, name, k, -h)
                fd_gpu[k] = (linear_loss(*gpu_eval(s, coeffs=cp), ct) -
                             linear_loss(*gpu_eval(s, coeffs=cm), ct)) / (2 * h)
                fd_orc[k] = (oracle_loss(cp) - oracle_loss(cm)) / (2 * h)
            scale = np.linalg.norm(got[name])
            assert np.max(np.abs(fd_gpu - got[name])) <= 1e-6 * scale, (name, fd_gpu, got[name])
            assert np.max(np.abs(fd_orc - got[name])) <= 1e-6 * scale, (name, fd_orc, got[name])
    finally:
        gpu_eval(s, coeffs=FE_FE)


def test_force_matching_autograd_knots(gpu_lib):
    """Force-matching loss over three configurations through EAMKnots on one
    shared system: loss.backward() against central differences of the loss."""
    configs = [fm_config(40 + c, n=6, sigma=0.1) for c in range(3)]
    # one system serves all three configurations: the state is set before each
    # forward, and each backward re-creates its own forward first
    s = MoldySystem.from_workload(configs[0], uselookup=True)
    refs = []
    for w in configs:
        s.set_state(x0=w.x0, b0=w.b0)
        _, f0, s0 = gpu_eval(s, coeffs=FE_FE)
        refs.append((f0, s0))
    rng = np.random.default_rng(2)
    theta = {k: torch.tensor(np.asarray(getattr(FE_FE, k)) * (1 + 1e-3 * rng.normal(size=len(getattr(FE_FE, k)))),
                             requires_grad=True) for k in adj.KNOT_NAMES}

    def loss_of(th):
        total = torch.zeros((), dtype=torch.float64)
        for w, (f0, s0) in zip(configs, refs):
            s.set_state(x0=w.x0, b0=w.b0)
            _, f, sig = adj.eam_knots(s, th)
            total = total + ((f - torch.as_tensor(f0)) ** 2).sum() + ((sig - torch.as_tensor(s0)) ** 2).sum()
        return total

    loss = loss_of(theta)
    loss.backward()
    h = 1e-6
    with torch.no_grad():
        for name in adj.KNOT_NAMES:
            g = theta[name].grad.numpy()
            fd = np.zeros(len(g))
            for k in range(len(g)):
                tp = {n: theta[n].detach().clone() for n in adj.KNOT_NAMES}
                tm = {n: theta[n].detach().clone() for n in adj.KNOT_NAMES}
                tp[name][k] += h
                tm[name][k] -= h
                fd[k] = (loss_of(tp).item() - loss_of(tm).item()) / (2 * h)
            assert np.max(np.abs(fd - g)) <= 1e-6 * np.linalg.norm(g), (name, fd, g)
    s.close()


def test_fused_force_matching_equals_per_configuration_autograd(gpu_lib):
    """ForceMatchingKnots (tables built once, each configuration evaluated
    once, the gradient formed in the forward pass) gives the loss and the
    knot gradient of the per-configuration EAMKnots path within 1e-11, with
    weights, and scales its gradient by the incoming one."""
    configs = [fm_config(60 + c, n=6, sigma=0.1) for c in range(3)]
    s = MoldySystem.from_workload(configs[0], uselookup=True)
    refs = []
    for w in configs:
        s.set_state(x0=w.x0, b0=w.b0)
        _, f0, s0 = gpu_eval(s, coeffs=FE_FE)
        refs.append((f0 + 1e-3, s0 * 1.01))
    rng = np.random.default_rng(5)
    base = {k: np.asarray(getattr(FE_FE, k)) * (1 + 1e-3 * rng.normal(size=len(getattr(FE_FE, k))))
            for k in adj.KNOT_NAMES}
    th1 = {k: torch.tensor(v, requires_grad=True) for k, v in base.items()}
    total = torch.zeros((), dtype=torch.float64)
    for w, (f0, s0) in zip(configs, refs):
        s.set_state(x0=w.x0, b0=w.b0)
        _, f, sig = adj.eam_knots(s, th1)
        total = total + 0.7 * ((f - torch.as_tensor(f0)) ** 2).sum() + 2.0 * ((sig - torch.as_tensor(s0)) ** 2).sum()
    total.backward()
    th2 = {k: torch.tensor(v, requires_grad=True) for k, v in base.items()}
    fused = adj.force_matching_knots(s, [(w.x0, w.b0) for w in configs], refs, th2, w_force=0.7, w_stress=2.0)
    (3.0 * fused).backward()
    assert abs(fused.item() - total.item()) <= 1e-11 * abs(total.item())
    for k in adj.KNOT_NAMES:
        a, b = th1[k].grad.numpy(), th2[k].grad.numpy() / 3.0
        assert np.max(np.abs(a - b)) <= 1e-11 * np.linalg.norm(a), (k, a, b)
    # two systems driven from two host threads: the same loss and gradient
    s2 = MoldySystem.from_workload(configs[0], uselookup=True)
    th3 = {k: torch.tensor(v, requires_grad=True) for k, v in base.items()}
    par = adj.force_matching_knots([s, s2], [(w.x0, w.b0) for w in configs], refs, th3, w_force=0.7, w_stress=2.0)
    par.backward()
    assert abs(par.item() - total.item()) <= 1e-11 * abs(total.item())
    for k in adj.KNOT_NAMES:
        a, b = th1[k].grad.numpy(), th3[k].grad.numpy()
        assert np.max(np.abs(a - b)) <= 1e-11 * np.linalg.norm(a), (k, a, b)
    s2.close()
    s.close()


def test_table_autograd_matches_reference(case):
    """EAMTables backward equals torch autograd of the restated forward."""
    w, o, s = case["w"], case["o"], case["s"]
    tt = {k: torch.tensor(v, requires_grad=True) for k, v in case["tabs"].items()}
    ct = cotangents(w.nm, seed=13)
    e, f, sig = adj.eam_tables(s, tt)
    (ct[0] * e + (torch.as_tensor(ct[1]) * f).sum() + (torch.as_tensor(ct[2]) * sig).sum()).backward()
    rt = torch_tables(case["tabs"])
    i, j = half_pairs(*o.nlist())
    st = o.get_state()
    e2, f2, s2 = eam_forward(st["x0"], st["b0"], i, j, w.atomic_mass, rt)
    (ct[0] * e2 + (torch.as_tensor(ct[1]) * f2).sum() + (torch.as_tensor(ct[2]) * s2).sum()).backward()
    for k in NAMES:
        assert rel_norm_err(tt[k].grad.numpy(), rt[k].grad.numpy()) <= 1e-9, k


def test_mixed_precision_handle_gives_fp64_gradients(case, gpu_lib):
    w = case["w"]
    ct = cotangents(w.nm)
    ref = case["s"].table_gradients(*ct)
    m = MoldySystem.from_workload(w, uselookup=True, precision="mixed")
    gpu_eval(m)
    got = m.table_gradients(*ct)
    m.close()
    for k in NAMES:
        assert rel_norm_err(got[k], ref[k]) <= 1e-10, k


def test_adjoint_order_and_mode_errors(gpu_lib):
    w = fm_config(1, n=5)
    s = MoldySystem.from_workload(w, uselookup=True)
    with pytest.raises(MoldyError) as ei:
        s.table_gradients(1.0)
    assert ei.value.code == 5
    gpu_eval(s)
    s.set_state(x0=w.x0 + 1e-4)
    with pytest.raises(MoldyError) as ei:
        s.table_gradients(1.0)
    assert ei.value.code == 5
    s.close()
    x = MoldySystem.from_workload(w, uselookup=False)
    gpu_eval(x)
    with pytest.raises(MoldyError) as ei:
        x.table_gradients(1.0)
    assert ei.value.code == 7
    x.close()


def test_batch_force_matching_equals_single_system_path(gpu_lib):
    """The batched force matching (every configuration in one MoldyBatch: one
    FP64 evaluation, the loss and the table adjoint on the device) gives the
    loss and the knot gradient of ForceMatchingKnots (one MoldySystem per
    configuration size, summed) within 1e-10 and 1e-8 (the pair sets are the
    same, the summation orders are not), on configurations of uneven size, and
    matches central differences (h = 1e-6) of its own loss within 1e-6."""
    from moldy_b200 import MoldyBatch
    configs = [fm_config(80 + c, n=n, sigma=0.1) for c, n in enumerate((6, 5, 6, 7, 5))]
    by_size = {}
    for c, w in enumerate(configs):
        by_size.setdefault(w.nm, []).append(c)
    systems = {nm: MoldySystem.from_workload(configs[cs[0]], uselookup=True) for nm, cs in by_size.items()}
    refs = [None] * len(configs)
    for nm, cs in by_size.items():
        for c in cs:
            w = configs[c]
            systems[nm].set_state(x0=w.x0, b0=w.b0)
            _, f0, s0 = gpu_eval(systems[nm], coeffs=FE_FE)
            refs[c] = (f0 + 1e-3, s0 * 1.01)
    rng = np.random.default_rng(6)
    base = {k: np.asarray(getattr(FE_FE, k)) * (1 + 1e-3 * rng.normal(size=len(getattr(FE_FE, k))))
            for k in adj.KNOT_NAMES}
    th1 = {k: torch.tensor(v, requires_grad=True) for k, v in base.items()}
    single = torch.zeros((), dtype=torch.float64)
    for nm, cs in by_size.items():
        single = single + adj.force_matching_knots(systems[nm], [(configs[c].x0, configs[c].b0) for c in cs],
                                                   [refs[c] for c in cs], th1, w_force=0.7, w_stress=2.0)
    single.backward()
    for sys_ in systems.values():
        sys_.close()
    b = MoldyBatch.from_workloads(configs)
    b.set_references([f for f, _ in refs], [sg for _, sg in refs])
    th2 = {k: torch.tensor(v, requires_grad=True) for k, v in base.items()}
    batched = adj.batch_force_matching_knots(b, th2, w_force=0.7, w_stress=2.0)
    batched.backward()
    assert abs(batched.item() - single.item()) <= 1e-10 * abs(single.item())
    for k in adj.KNOT_NAMES:
        a, g = th1[k].grad.numpy(), th2[k].grad.numpy()
        assert np.max(np.abs(a - g)) <= 1e-8 * np.linalg.norm(a), (k, a, g)

    def loss_of(th):
        return adj.batch_force_matching_knots(b, th, w_force=0.7, w_stress=2.0).item()

    h = 1e-6
    for name in adj.KNOT_NAMES:
        g = th2[name].grad.numpy()
        fd = np.zeros_like(g)
        for k in range(len(g)):
            tp = {n: torch.tensor(base[n]) for n in adj.KNOT_NAMES}
            tm = {n: torch.tensor(base[n]) for n in adj.KNOT_NAMES}
            tp[name][k] += h
            tm[name][k] -= h
            fd[k] = (loss_of(tp) - loss_of(tm)) / (2 * h)
        assert np.max(np.abs(fd - g)) <= 1e-6 * np.linalg.norm(g), (name, fd, g)
    b.close()
