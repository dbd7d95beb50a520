"""Pins of the CPU oracle (no GPU): known answers for the FETRANSMETAL Fe-Fe
potential and structural properties of the link cells and the half list."""
import json
import os

import numpy as np
import pytest

from moldy_b200 import workloads as wl
from tests.helpers import pair_set, real_forces

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _perfect(oracle_mod, a0, lookup, n=4):
    w = wl.make_workload(n, a0=a0, sigma=0.0, temperature=0.0, ivol=1)
    o = oracle_mod.from_workload(w, uselookup=lookup, threads=1)
    o.force()
    return w, o


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLDEN, "perfect_lattice.json")))["cases"])
def test_perfect_lattice_exact(oracle_mod, case):
    """Exact-mode energy and density equal the 30-digit analytic values."""
    w, o = _perfect(oracle_mod, case["a0"], lookup=False)
    fo = o.force_out()
    d = o.density()
    assert abs(fo["pe"] / w.nm - case["e_per_atom"]) < 1e-12
    assert np.max(np.abs(d["rho"] - case["rho"])) < 1e-11
    # every atom sits at a centre of inversion: zero force, zero shear virial
    assert np.max(np.abs(real_forces(o.forces(), w.b0))) < 1e-12
    tp = fo["tp"]
    assert np.max(np.abs(tp - np.diag(np.diag(tp)))) < 1e-10
    assert abs(tp[0, 0] - tp[1, 1]) < 1e-9 and abs(tp[1, 1] - tp[2, 2]) < 1e-9


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLDEN, "perfect_lattice.json")))["cases"])
def test_perfect_lattice_virial_is_de_dvolume(oracle_mod, case):
    """tp is the configurational virial.  tp(a,b) = sum r_a d_b fp with d = r / L
    (cubic box of n cells, L = n a0) and fp = -(dE/dr)/r, so tr(tp) = -sum r dE/dr / L,
    while a uniform stretch gives a dE/da = sum r dE/dr: dE/da = -n tr(tp)."""
    n = 4
    w, o = _perfect(oracle_mod, case["a0"], lookup=False, n=n)
    tp = o.force_out()["tp"]
    de_da = -n * np.trace(tp)
    assert abs(de_da / w.nm - case["de_da_per_atom"]) < 1e-11


def test_perfect_lattice_lookup_error_bound(oracle_mod):
    """Lookup mode differs from exact only by the interpolation error of the
    tables; the embedding table has a step of 2 in rho, which dominates."""
    case = json.load(open(os.path.join(GOLDEN, "perfect_lattice.json")))["cases"][0]
    w, o = _perfect(oracle_mod, case["a0"], lookup=True)
    e = o.force_out()["pe"] / w.nm
    rho = case["rho"]
    # linear interpolation error of -sqrt on [24, 26]: |F''| h^2 / 8 = rho^-1.5 / 4 * 4 / 8
    bound = 0.25 * (24.0 ** -1.5) * 4.0 / 8.0 * 1.05
    assert abs(e - case["e_per_atom"]) < bound + 1e-6
    assert abs(o.density()["rho"][0] - rho) < 1e-5


def test_tables_zero_beyond_cutoff(oracle_mod):
    w = wl.make_workload(3, sigma=0.0, temperature=0.0)
    o = oracle_mod.from_workload(w, uselookup=True)
    t = o.tables()
    nz = [np.nonzero(t[k])[0].max() for k in ("vee", "dvee", "phi", "dphi")]
    # last nonzero node: phi/dphi at 3.726 A (node 3105), vee/dvee below 3.38247 A
    assert max(nz) == 3105
    assert nz[0] == nz[1] == 2818
    assert np.isinf(t["vee"][0])            # Biersack 1/r at r = 0
    assert t["emb"][0] == 0.0 and np.signbit(t["emb"][0])


def test_fetm_setup_constants(oracle_mod):
    w = wl.make_workload(3, sigma=0.0, temperature=0.0)
    o = oracle_mod.from_workload(w, uselookup=False)
    d = o.fetm_derived()
    assert d["bier_cut1"] == float(np.float32(0.9))
    assert d["bier_cut2"] == float(np.float32(1.9))
    # phi is flat below its maximum; its slope changes sign there
    pc = d["phi_cut1"]
    assert 1.7 < pc < 1.9
    assert o.src(3, pc + 1e-6) < 0.0 < -o.src(3, pc + 1e-6) + 1.0
    # join continuity: the log-Hermite join meets both ends
    assert abs(o.src(0, d["bier_cut2"] - 1e-9) - d["sc3"]) < 1e-6 * abs(d["sc3"])
    assert abs(o.src(0, d["bier_cut1"] + 1e-9) - d["sc1"]) < 1e-6 * abs(d["sc1"])


def test_force_is_minus_energy_gradient(oracle_mod):
    """Exact mode: central differences of the potential energy reproduce the
    real forces B0 f (and the embedding term) to FD accuracy."""
    w = wl.make_workload(3, sigma=0.12, temperature=0.0, ivol=1, seed=7)
    binv = np.linalg.inv(w.b0)

    def energy(x0):
        w2 = w.copy()
        w2.x0 = x0
        o = oracle_mod.from_workload(w2, uselookup=False, threads=1)
        o.force()
        return o.force_out()["pe"], o

    e0, o = energy(w.x0)
    f = real_forces(o.forces(), w.b0)
    h = 1e-5
    rng = np.random.default_rng(3)
    for a in rng.choice(w.nm, size=6, replace=False):
        for k in range(3):
            d = np.zeros(3)
            d[k] = h
            xp = w.x0.copy(); xp[a] += binv @ d
            xm = w.x0.copy(); xm[a] -= binv @ d
            fd = -(energy(xp)[0] - energy(xm)[0]) / (2 * h)
            assert abs(fd - f[a, k]) < 2e-6, (a, k, fd, f[a, k])


def test_lookup_forces_close_to_exact(oracle_mod):
    w = wl.make_workload(4, sigma=0.08, temperature=0.0, seed=11)
    o1 = oracle_mod.from_workload(w, uselookup=False, threads=1)
    o2 = oracle_mod.from_workload(w, uselookup=True, threads=1)
    o1.force(); o2.force()
    f1 = real_forces(o1.forces(), w.b0)
    f2 = real_forces(o2.forces(), w.b0)
    rms = np.sqrt(np.mean((f1 - f2) ** 2))
    assert rms < 5e-3


def test_linkup_chains(oracle_mod):
    w = wl.make_workload(6, sigma=0.1, temperature=0.0, seed=5)
    o = oracle_mod.from_workload(w)
    l0, link, ic = o.linkcells()
    nlc = w.nlc
    seen = np.zeros(w.nm + 1, dtype=int)
    for c, start in enumerate(l0, start=1):
        if start == 0:
            continue
        chain = [start]
        j = link[start - 1]
        while j != start:
            chain.append(j)
            j = link[j - 1]
        assert chain == sorted(chain)            # linkup inserts in index order
        for a in chain:
            assert ic[a - 1] == c
            seen[a] += 1
    assert np.all(seen[1:] == 1)
    # cell index from the fractional coordinate
    s = w.x0 - np.round(w.x0) + 0.4999999999
    cells = (s * np.array(nlc)).astype(int)
    ref = cells[:, 0] + nlc[0] * cells[:, 1] + nlc[0] * nlc[1] * cells[:, 2] + 1
    assert np.array_equal(ref, ic)


def test_relink_keeps_cell_membership(oracle_mod):
    """relink after moves gives the same cell membership as a fresh linkup."""
    w = wl.make_workload(6, sigma=0.0, temperature=0.0, seed=5)
    o = oracle_mod.from_workload(w)
    rng = np.random.default_rng(9)
    x = w.x0 + rng.uniform(-0.06, 0.06, size=w.x0.shape)
    o.set_state(x, w.x1, w.x2, w.b0, w.b1, w.b2, w.atomic_number, w.atomic_mass, w.del2)
    o.relink()
    l0, link, ic = o.linkcells()
    o2 = oracle_mod.from_workload(w)
    o2.set_state(x, w.x1, w.x2, w.b0, w.b1, w.b2, w.atomic_number, w.atomic_mass, w.del2)
    o2.linkup()
    l0b, linkb, icb = o2.linkcells()
    assert np.array_equal(ic, icb)


def test_half_list_is_all_pairs_within_rnear(oracle_mod):
    """With 3 link cells per side the half stencil covers every pair once, so
    the half list is exactly the set of minimum-image pairs closer than rnear."""
    w = wl.make_workload(4, sigma=0.1, temperature=0.0, seed=2)
    assert w.nlc == (3, 3, 3)
    o = oracle_mod.from_workload(w)
    assert o.update_neighbourlist() == 0
    nl, nn = o.nlist()
    got = pair_set(nl, nn)
    d = w.x0[:, None, :] - w.x0[None, :, :]
    d -= np.round(d)
    r = np.linalg.norm(d @ w.b0.T, axis=2)
    iu = np.triu_indices(w.nm, 1)
    mask = r[iu] < w.rnear
    want = {(int(i) + 1, int(j) + 1) for i, j in zip(iu[0][mask], iu[1][mask])}
    assert got == want
    assert len(got) == int(nn.sum())          # no pair listed twice


def test_neighbour_overflow_is_reported(oracle_mod):
    w = wl.make_workload(4, sigma=0.0, temperature=0.0)
    w.nnbrs = 10
    o = oracle_mod.from_workload(w)
    assert o.update_neighbourlist() == 1


def test_nve_energy_conservation_exact(oracle_mod):
    """Velocity Verlet in exact mode conserves the total energy of a small
    300 K crystal to well below the kinetic-energy fluctuation."""
    w = wl.make_workload(4, sigma=0.05, temperature=300.0, ivol=1, seed=4, nbrupdate=10)
    o = oracle_mod.from_workload(w, uselookup=False, threads=1)
    o.md_init()
    te = [o.md_step()["te"] for _ in range(60)]
    assert np.ptp(te) / w.nm < 2e-5


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLDEN, "perfect_lattice.json")))["cases"])
def test_quench_reaches_perfect_lattice_energy(oracle_mod, case):
    """VA14CD + derivs (exact mode) from a displaced lattice at a fixed box
    ends at the 30-digit perfect-lattice energy."""
    w = wl.make_workload(4, a0=case["a0"], sigma=0.1, temperature=0.0, ivol=1, seed=7)
    o = oracle_mod.from_workload(w, uselookup=False, threads=2)
    q = o.quench(maxfn=5000, criterion=1, fmax=1e-6)
    assert q["iflag"] == 0 and q["fmax"] <= 1e-6
    assert abs(q["f"] / w.nm - case["e_per_atom"]) < 1e-12


def test_quench_reference_criterion(oracle_mod):
    """The reference's acceptance test: sum of squared gradient <= 5e-7 nm."""
    rng = np.random.default_rng(3)
    w = wl.make_workload(5, sigma=0.1, temperature=0.0, ivol=1, seed=3,
                         strain=wl.random_symmetric_strain(rng, 0.02))
    o = oracle_mod.from_workload(w, uselookup=True, threads=2)
    o.force()
    e0 = float(o.energy_calc().sum())
    q = o.quench(maxfn=5000, criterion=0)
    assert q["iflag"] == 0
    assert q["gsumsq"] <= 5e-7 * w.nm
    assert q["f"] < e0
