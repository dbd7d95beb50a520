"""Adjoint checks that need no GPU: the torch FP64 reference forward against
the oracle, the knot contraction against finite differences of the table
builder, and the sharded gradient all-reduce on two gloo ranks."""
import os

import numpy as np
import pytest
import torch

from moldy_b200 import FE_FE, FeFeCoefficients
from moldy_b200 import adjoint as adj
from moldy_b200 import workloads as wl
from tests.eam_torch import NAMES, eam_forward, half_pairs, torch_tables
from tests.helpers import real_forces, rel_norm_err


@pytest.fixture(scope="module")
def host_lib():
    from moldy_b200 import _lib, build
    build.build()
    return _lib.load()


def fm_config(seed: int, n: int = 6, sigma: float = 0.12):
    rng = np.random.default_rng(seed)
    return wl.make_workload(n, sigma=sigma, temperature=0.0, ivol=1, seed=seed,
                            strain=wl.random_symmetric_strain(rng, 0.03))


def oracle_pairs(oracle_mod, w):
    o = oracle_mod.from_workload(w, uselookup=True, threads=1)
    o.force()
    nl, nn = o.nlist()
    return o, half_pairs(nl, nn)


def test_torch_reference_matches_oracle(oracle_mod):
    """The torch restatement reproduces the oracle's E, F and sigma (1e-10)."""
    w = fm_config(3)
    o, (i, j) = oracle_pairs(oracle_mod, w)
    st = o.get_state()
    tabs = torch_tables(o.tables(), requires_grad=False)
    e, f, s = eam_forward(st["x0"], st["b0"], i, j, w.atomic_mass, tabs, ivol=w.ivol)
    fo = o.force_out()
    f_or = real_forces(o.forces(), st["b0"])
    s_or = -(fo["tp"] @ st["b0"].T) / fo["vol"]
    assert abs(e.item() - fo["pe"]) <= 1e-10 * abs(fo["pe"])
    assert rel_norm_err(f.numpy(), f_or) <= 1e-10
    assert rel_norm_err(s.numpy(), s_or) <= 1e-10


def test_host_tables_match_oracle(oracle_mod, host_lib):
    """moldy_fetm_build_tables is bit-identical to the oracle's tables."""
    o = oracle_mod.Oracle(16, nnbrs=8, ivol=1, ntcm=1)
    o.set_fetm(FE_FE.av, FE_FE.rv, FE_FE.ap, FE_FE.rp)
    o.set_lookup(True, 5000)
    ref = o.tables()
    got = adj.fetm_tables(FE_FE, 5000)
    for k in NAMES:
        assert np.array_equal(got[k], ref[k]), k


def _shift(coeffs, name, k, h):
    d = {f: np.array(getattr(coeffs, f), dtype=np.float64) for f in ("av", "rv", "ap", "rp")}
    d[name][k] += h
    return FeFeCoefficients(**d)


def test_knot_vjp_matches_finite_differences(host_lib):
    """g . dT/dtheta from the contraction agrees with central differences
    (h = 1e-6) of the table builder, for a random cotangent g on every node."""
    n = 5000
    rng = np.random.default_rng(11)
    g = {k: rng.normal(size=n + 1) for k in NAMES}
    vjp = adj.fetm_knot_vjp(FE_FE, g, n)
    h = 1e-6
    for name in adj.KNOT_NAMES:
        fd = np.zeros(len(vjp[name]))
        for k in range(len(fd)):
            tp = adj.fetm_tables(_shift(FE_FE, name, k, h), n)
            tm = adj.fetm_tables(_shift(FE_FE, name, k, -h), n)
            # vee(0) is the Biersack singularity: identical infinities in both
            fd[k] = sum(float(g[t] @ np.where(np.isfinite(tp[t]), tp[t] - tm[t], 0.0)) for t in NAMES) / (2 * h)
        err = np.abs(fd - vjp[name]) / max(np.linalg.norm(vjp[name]), 1e-300)
        assert err.max() <= 1e-6, (name, fd, vjp[name])


def test_shard_configs_balanced():
    natoms = [1024] * 200 + [2000] * 37 + [128] * 19
    for ws in (1, 2, 3, 8):
        shards = adj.shard_configs(natoms, ws)
        assert sorted(c for s in shards for c in s) == list(range(len(natoms)))
        loads = [sum(natoms[c] for c in s) for s in shards]
        assert max(loads) - min(loads) <= max(natoms)


def _fm_table_grad(oracle_mod, configs, tabs0, tabs):
    """Force-matching loss against tabs0 and its table gradient (torch autograd)."""
    grads = {k: torch.zeros(len(tabs[k]), dtype=torch.float64) for k in NAMES}
    total = 0.0
    for w in configs:
        o, (i, j) = oracle_pairs(oracle_mod, w)
        st = o.get_state()
        _, f0, s0 = eam_forward(st["x0"], st["b0"], i, j, w.atomic_mass, torch_tables(tabs0, False))
        tt = torch_tables(tabs)
        _, f, s = eam_forward(st["x0"], st["b0"], i, j, w.atomic_mass, tt)
        loss = ((f - f0) ** 2).sum() + ((s - s0) ** 2).sum()
        loss.backward()
        total += loss.item()
        for k in NAMES:
            if tt[k].grad is not None:   # emb enters E only
                grads[k] += tt[k].grad
    return total, grads


def _perturbed_tables(tabs0, seed=5):
    rng = np.random.default_rng(seed)
    return {k: tabs0[k] * (1.0 + 1e-3 * rng.normal(size=len(tabs0[k]))) for k in NAMES}


def _rank_main(rank, world, port, configs, tabs0, tabs, out_path):
    import torch.distributed as dist
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shards = adj.shard_configs([w.nm for w in configs], world)
        mine = [configs[c] for c in shards[rank]]
        _, g = _fm_table_grad(oracle, mine, tabs0, tabs)
        flat = [g[k] for k in NAMES]
        adj.allreduce_gradients(flat)
        if rank == 0:
            np.save(out_path, torch.cat(flat).numpy())
    finally:
        dist.destroy_process_group()


def test_sharded_gradient_allreduce_gloo(oracle_mod, tmp_path):
    """Two gloo ranks each take a shard of the configurations; the summed
    gradient equals the serial one (to rounding of the summation order)."""
    import socket
    import torch.multiprocessing as mp
    configs = [fm_config(20 + c, n=5, sigma=0.1) for c in range(4)]
    o = oracle_mod.Oracle(16, nnbrs=8, ivol=1, ntcm=1)
    o.set_fetm(FE_FE.av, FE_FE.rv, FE_FE.ap, FE_FE.rp)
    o.set_lookup(True, 5000)
    tabs0 = o.tables()
    tabs = _perturbed_tables(tabs0)
    _, g_serial = _fm_table_grad(oracle_mod, configs, tabs0, tabs)
    serial = torch.cat([g_serial[k] for k in NAMES]).numpy()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "g.npy")
    mp.start_processes(_rank_main, args=(2, port, configs, tabs0, tabs, out), nprocs=2,
                       join=True, start_method="spawn")
    got = np.load(out)
    assert rel_norm_err(got, serial) <= 1e-12
