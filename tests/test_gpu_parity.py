"""GPU parity tests: libmoldy_gpu.so (through its C ABI) against the CPU oracle
on the same seeded inputs.

Tolerances:
* link cells, neighbour lists: bit-exact (same l0/link/ic, same NLIST/NUMN);
* lookup tables: bit-exact (same host build, same arithmetic order);
* forces, density, energy, virial of one FP64 force call: norm-wise relative
  error <= 1e-10 (the sums run in another order, with FP64 atomics);
* trajectories: differences grow from the last bit, so 100 steps are checked
  against the oracle with a looser, stated bound.
"""
import numpy as np
import pytest

from moldy_b200 import workloads as wl
from tests.helpers import real_forces, rel_norm_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _pair(oracle_mod, gpu_lib, w, *, uselookup=True, precision="fp64"):
    from moldy_b200 import MoldySystem
    o = oracle_mod.from_workload(w, uselookup=uselookup, threads=1)
    g = MoldySystem.from_workload(w, uselookup=uselookup, precision=precision)
    return o, g


def test_tables_bit_exact(oracle_mod, gpu_lib):
    w = wl.make_workload(3, sigma=0.0, temperature=0.0)
    o, g = _pair(oracle_mod, gpu_lib, w)
    to, tg = o.tables(), g.tables()
    for k in to:
        assert np.array_equal(to[k], tg[k], equal_nan=True), k


@pytest.mark.parametrize("n,sigma,seed", [(10, 0.05, 1), (4, 0.1, 2), (7, 0.2, 3)])
def test_linkup_and_neighbour_list_exact(oracle_mod, gpu_lib, n, sigma, seed):
    w = wl.make_workload(n, sigma=sigma, temperature=0.0, seed=seed)
    o, g = _pair(oracle_mod, gpu_lib, w)
    g.linkup()
    lo = o.linkcells()
    lg = g.linkcells(o.ncell)
    for a, b in zip(lo, lg):
        assert np.array_equal(a, b)
    assert o.update_neighbourlist() == 0
    g.update_neighbourlist()
    nlo, nno = o.nlist()
    nlg, nng = g.neighbour_list()
    assert np.array_equal(nno, nng)
    for i in range(w.nm):
        assert np.array_equal(nlo[i, :nno[i]], nlg[i, :nng[i]]), i


def test_strained_box_neighbour_list_exact(oracle_mod, gpu_lib):
    rng = np.random.default_rng(4)
    w = wl.make_workload(9, sigma=0.1, temperature=0.0, seed=4,
                         strain=wl.random_symmetric_strain(rng, 0.02))
    o, g = _pair(oracle_mod, gpu_lib, w)
    g.linkup()
    assert o.update_neighbourlist() == 0
    g.update_neighbourlist()
    nlo, nno = o.nlist()
    nlg, nng = g.neighbour_list()
    assert np.array_equal(nno, nng)
    mask = np.arange(w.nnbrs)[None, :] < nno[:, None]
    assert np.array_equal(nlo[mask], nlg[mask])


@pytest.mark.parametrize("n,nlc", [(10, 3), (10, 4), (12, 4), (12, 3)])
def test_neighbour_list_exact_beyond_staging(oracle_mod, gpu_lib, n, nlc):
    """Few, crowded link cells: 31 to 128 atoms per cell on average, so the
    14 cells of a home cell's half stencil hold more than the 384 candidates
    the builder stages in shared memory (the rest are read from global
    memory), and home cells of
    more than 32 atoms take several rounds of lanes; 3 cells per direction use
    the fixed-point pre-test, 4 the cell-relative one.  NLIST/NUMN are still
    identical entry by entry."""
    w = wl.make_workload(n, sigma=0.1, temperature=0.0, seed=14)
    w.nlc = (nlc, nlc, nlc)
    o, g = _pair(oracle_mod, gpu_lib, w)
    g.linkup()
    counts = np.bincount(g.linkcells(nlc ** 3)[2] - 1, minlength=nlc ** 3)
    assert counts.mean() * 14 > 384
    assert o.update_neighbourlist() == 0
    g.update_neighbourlist()
    nlo, nno = o.nlist()
    nlg, nng = g.neighbour_list()
    assert np.array_equal(nno, nng)
    for i in range(w.nm):
        assert np.array_equal(nlo[i, :nno[i]], nlg[i, :nng[i]]), i


# (dx, dy, dz) of the 13 cells of the half stencil after the home cell, in
# the reference's loop order (src/neighbourlist_m.F90:103-276); the reverse
# rows walk their negations
_HALF = [(1, 0, 0), (-1, 1, 0), (0, 1, 0), (1, 1, 0), (-1, -1, 1), (0, -1, 1), (1, -1, 1),
         (-1, 0, 1), (0, 0, 1), (1, 0, 1), (-1, 1, 1), (0, 1, 1), (1, 1, 1)]


def _expected_reverse_rows(g, w, nlc):
    """The transpose of NLIST, each row ordered as the build stages its
    candidates: the own cell (chain order) before the atom, then the mirror
    cells -offset(1) ... -offset(13), each in chain order."""
    ncell = nlc[0] * nlc[1] * nlc[2]
    l0, link, ic = g.linkcells(ncell)
    chain = np.zeros(w.nm, dtype=np.int64)
    for c in range(ncell):
        # the chain is circular: the last atom links back to the head
        a, k = l0[c], 0
        while a and k < w.nm:
            chain[a - 1] = k
            k += 1
            a = link[a - 1]
            if a == l0[c]:
                break
    cell = ic - 1
    cxyz = np.stack([cell % nlc[0], (cell // nlc[0]) % nlc[1], cell // (nlc[0] * nlc[1])], axis=1)
    mirror = {}
    for k, (dx, dy, dz) in enumerate(_HALF):
        mirror[((-dx) % nlc[0], (-dy) % nlc[1], (-dz) % nlc[2])] = 1 + k
    nl, nn = g.neighbour_list()
    rows = [[] for _ in range(w.nm)]
    for j in range(w.nm):
        for i in nl[j, :nn[j]] - 1:
            rows[i].append(j)
    out = []
    for i in range(w.nm):
        def key(j, i=i):
            off = tuple(int(v) for v in (cxyz[j] - cxyz[i]) % np.array(nlc))
            return (0 if off == (0, 0, 0) else mirror[off], chain[j])
        out.append(sorted(rows[i], key=key))
    return out


@pytest.mark.parametrize("n,nlc,strain", [(10, None, False), (9, None, True), (10, 3, False), (12, 4, False),
                                          (12, 3, False)])
def test_reverse_rows_are_the_ordered_transpose(gpu_lib, n, nlc, strain):
    """The reverse rows formed with the half list hold, for every atom i,
    exactly the atoms j with i in NLIST(:, j), in staging order (own cell,
    then the mirror cells, each in chain order); covers the cell-relative
    pre-test (default cells, a strained box), the fixed-point one (3 cells per
    direction), candidates beyond the staging (12^3 bcc in 4^3 cells: 2 and 3
    rounds of home atoms) and cells fuller than the reverse-row masks hold
    (12^3 bcc in 3^3 cells, 128 atoms per cell: the scatter-and-sort path)."""
    rng = np.random.default_rng(21)
    w = wl.make_workload(n, sigma=0.1, temperature=0.0, seed=22,
                         strain=wl.random_symmetric_strain(rng, 0.02) if strain else None)
    if nlc is not None:
        w.nlc = (nlc, nlc, nlc)
    from moldy_b200 import MoldySystem
    g = MoldySystem.from_workload(w, precision="mixed")
    g.linkup()
    g.update_neighbourlist()
    exp = _expected_reverse_rows(g, w, tuple(w.nlc))
    rl, nr = g.reverse_list()
    assert np.array_equal(nr, [len(r) for r in exp])
    for i in range(w.nm):
        assert np.array_equal(rl[i, :nr[i]] - 1, exp[i]), i
    g.close()


@pytest.mark.parametrize("n", [8, 30])
def test_relink_chain_order_exact(oracle_mod, gpu_lib, n):
    """relink replays the reference's chain surgery: same l0/link after moves,
    and the following neighbour list is identical entry by entry (n=30 has
    13^3 = 2197 link cells, more than one thread block of cells)."""
    w = wl.make_workload(n, sigma=0.05, temperature=0.0, seed=6)
    o, g = _pair(oracle_mod, gpu_lib, w)
    g.linkup()
    rng = np.random.default_rng(12)
    x = w.x0.copy()
    for _ in range(3):
        x = x + rng.normal(0.0, 0.02, size=x.shape)
        o.set_state(x, w.x1, w.x2, w.b0, w.b1, w.b2, w.atomic_number, w.atomic_mass, w.del2)
        g.set_state(x0=x)
        o.relink()
        g.relink()
        lo = o.linkcells()
        lg = g.linkcells(o.ncell)
        for a, b in zip(lo, lg):
            assert np.array_equal(a, b)
    assert o.update_neighbourlist() == 0
    g.update_neighbourlist()
    nlo, nno = o.nlist()
    nlg, nng = g.neighbour_list()
    assert np.array_equal(nno, nng)
    mask = np.arange(w.nnbrs)[None, :] < nno[:, None]
    assert np.array_equal(nlo[mask], nlg[mask])


@pytest.mark.parametrize("uselookup", [True, False])
@pytest.mark.parametrize("ivol", [1, 0])
def test_force_fp64(oracle_mod, gpu_lib, uselookup, ivol):
    w = wl.make_workload(10, sigma=0.05, temperature=300.0, ivol=ivol, seed=1)
    o, g = _pair(oracle_mod, gpu_lib, w, uselookup=uselookup)
    o.force()
    fg = g.force()
    fo = o.force_out()
    assert rel_norm_err(g.forces(), o.forces()) < FP64_TOL
    do, dg = o.density(), g.density()
    for k in ("rho", "afrho", "dafrho"):
        assert rel_norm_err(dg[k], do[k]) < FP64_TOL, k
    assert abs(fg["pe"] - fo["pe"]) < FP64_TOL * abs(fo["pe"])
    for k in ("tp", "tk", "tc", "tg", "tgdot", "fb"):
        assert rel_norm_err(fg[k], fo[k]) < FP64_TOL, k
    assert abs(fg["vol"] - fo["vol"]) < 1e-12 * fo["vol"]
    assert fg["ntc"] == o.ntc and fg["rebuilt"]


def test_force_perfect_lattice_zero(oracle_mod, gpu_lib):
    import json, os
    case = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                       "perfect_lattice.json")))["cases"][0]
    w = wl.make_workload(6, a0=case["a0"], sigma=0.0, temperature=0.0)
    _, g = _pair(oracle_mod, gpu_lib, w, uselookup=False)
    fg = g.force()
    assert abs(fg["pe"] / w.nm - case["e_per_atom"]) < 1e-12
    assert np.max(np.abs(real_forces(g.forces(), w.b0))) < 1e-11


def test_atomstress_and_energy_calc(oracle_mod, gpu_lib):
    w = wl.make_workload(6, sigma=0.08, temperature=0.0, seed=8, atomstress=1)
    o, g = _pair(oracle_mod, gpu_lib, w)
    o.force()
    g.force()
    assert rel_norm_err(g.atomstress(), o.atomstress()) < FP64_TOL
    assert rel_norm_err(g.energy_calc(), o.energy_calc()) < FP64_TOL


def test_set_tables_drop_in(oracle_mod, gpu_lib):
    """Tables handed over by the caller (potential_set_lookup output) give the
    same forces as the built-in FETRANSMETAL set-up."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(6, sigma=0.08, temperature=0.0, seed=9)
    o = oracle_mod.from_workload(w, uselookup=True, threads=1)
    o.force()
    g = MoldySystem(w.nm, rnear=w.rnear, deltat=w.deltat, ivol=w.ivol, ntcm=w.ntcm, nlc=w.nlc)
    g.set_tables(o.tables())
    g.set_state(w.x0, w.x1, w.x2, w.b0, w.b1, w.b2, w.atomic_number, w.atomic_mass, w.del2)
    g.force()
    assert rel_norm_err(g.forces(), o.forces()) < FP64_TOL


def _offset_tables(o, nlookup, rmin, rmax):
    """Caller tables over [rmin, rmax] from the analytic FETRANSMETAL Fe-Fe
    functions: rmin > 0, and since rmax lies inside the cut, the last node is
    nonzero, so every pair beyond rmax takes T(nlookup) (src/lookup_m.F90:322-340)."""
    r = rmin + np.arange(nlookup + 1) * ((rmax - rmin) / nlookup)
    t = {k: np.array([o.src(i, x) for x in r]) for i, k in enumerate(("vee", "dvee", "phi", "dphi"))}
    full = o.tables()
    t["emb"], t["demb"] = full["emb"], full["demb"]
    return t


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_set_tables_offset_range_nonzero_tail(oracle_mod, gpu_lib, precision):
    """Caller tables with rmin = 1.2 A and rmax = 3.2 A (inside the 3.73 A cut,
    so the last node is nonzero and every listed pair out to rnear contributes):
    FP64 within 1e-10 of the oracle; mixed within the accuracy gate (real-force
    RMS <= 1e-5 eV/A, pe <= 1e-6 eV/atom, stress <= 1e-4 GPa)."""
    from moldy_b200 import MoldySystem
    from moldy_b200 import units
    w = wl.make_workload(6, sigma=0.08, temperature=0.0, seed=9)
    o = oracle_mod.from_workload(w, uselookup=True, threads=1)
    rmin, rmax = 1.2, 3.2
    tabs = _offset_tables(o, 5000, rmin, rmax)
    assert min(abs(tabs[k][-1]) for k in ("vee", "dvee", "phi", "dphi")) > 1e-3
    o.set_tables(tabs, rmin=rmin, rmax=rmax)
    o.force()
    oo = o.force_out()
    g = MoldySystem(w.nm, rnear=w.rnear, deltat=w.deltat, ivol=w.ivol, ntcm=w.ntcm, nlc=w.nlc,
                    precision=precision)
    g.set_tables(tabs, rmin=rmin, rmax=rmax)
    g.set_state(w.x0, w.x1, w.x2, w.b0, w.b1, w.b2, w.atomic_number, w.atomic_mass, w.del2)
    go = g.force()
    if precision == "fp64":
        assert rel_norm_err(g.forces(), o.forces()) < FP64_TOL
        assert rel_norm_err(g.density()["rho"], o.density()["rho"]) < FP64_TOL
        assert abs(go["pe"] - oo["pe"]) < FP64_TOL * abs(oo["pe"])
        assert rel_norm_err(go["tp"], oo["tp"]) < FP64_TOL
        return
    df = real_forces(g.forces(), w.b0) - real_forces(o.forces(), w.b0)
    rms = float(np.sqrt(np.mean(np.sum(df * df, axis=1))))
    assert rms <= 1e-5, rms
    assert abs(go["pe"] - oo["pe"]) / w.nm < 1e-6
    sig = lambda fo: -(w.b0 @ (fo["tp"]).T).T / fo["vol"] * units.PRESS_TO_GPA
    assert np.max(np.abs(sig(go) - sig(oo))) < 1e-4


def test_md_trajectory_nve_100_steps(oracle_mod, gpu_lib):
    """2000-atom bcc Fe, 300 K, NVE, dt 1 fs, 100 steps (lookup tables)."""
    w = wl.config_small_nve()
    o, g = _pair(oracle_mod, gpu_lib, w)
    o.md_init()
    g.md_init()
    th_o = [o.md_step() for _ in range(100)]
    th_g = g.md_steps(100)
    for k in ("pe", "ke", "te"):
        a = np.array([t[k] for t in th_o])
        b = np.array([t[k] for t in th_g])
        assert np.max(np.abs(a - b)) < 1e-7 * w.nm, k
    so, sg = o.get_state(), g.get_state()
    dx = (sg["x0"] - so["x0"]) @ w.b0.T
    assert np.max(np.abs(dx)) < 1e-8          # Angstrom after 100 fs
    assert [t["ntc"] for t in th_g] == [int(t["ntc"]) for t in th_o]


def test_md_trajectory_npt_box(oracle_mod, gpu_lib):
    """Parrinello-Rahman NPT (ivol=0) at 1200 K: box matrices follow the oracle."""
    w = wl.make_workload(6, sigma=0.05, temperature=1200.0, ivol=0, seed=21, nbrupdate=7)
    o, g = _pair(oracle_mod, gpu_lib, w)
    o.md_init()
    g.md_init()
    th_o = [o.md_step() for _ in range(30)]
    th_g = g.md_steps(30)
    so, sg = o.get_state(), g.get_state()
    assert rel_norm_err(sg["b0"], so["b0"]) < 1e-11
    assert rel_norm_err(sg["b1"], so["b1"]) < 1e-6
    assert abs(th_g[-1]["vol"] - th_o[-1]["vol"]) < 1e-9 * th_o[-1]["vol"]
    assert abs(th_g[-1]["th"] - th_o[-1]["th"]) < 1e-8 * abs(th_o[-1]["th"])


def test_velocityverlet_single_step_matches(oracle_mod, gpu_lib):
    w = wl.make_workload(6, sigma=0.05, temperature=600.0, ivol=0, seed=31, nbrupdate=3)
    o, g = _pair(oracle_mod, gpu_lib, w)
    o.md_init()
    g.md_init()
    for _ in range(4):
        o.velocityverlet()
        g.velocityverlet()
        so, sg = o.get_state(), g.get_state()
        for k in ("x0", "x1", "x2"):
            assert rel_norm_err(sg[k], so[k]) < 1e-9, k
        s_o = o.update_therm_avs()
        s_g = g.update_therm_avs()
        assert np.allclose(s_g, s_o, rtol=1e-9, atol=0)


def test_neighbour_overflow_error(oracle_mod, gpu_lib):
    from moldy_b200 import MoldyError
    w = wl.make_workload(4, sigma=0.0, temperature=0.0)
    w.nnbrs = 12
    _, g = _pair(oracle_mod, gpu_lib, w)
    with pytest.raises(MoldyError) as ei:
        g.force()
    assert ei.value.code == 2


def test_md_many_rebuilds_large_box(oracle_mod, gpu_lib):
    """54,000 atoms (13^3 link cells), NPT 1200 K, rebuild every 3 steps: after
    12 steps (4 relinks, 5 list builds) thermo, link cells and the neighbour
    list still follow the oracle."""
    w = wl.make_workload(30, sigma=0.05, temperature=1200.0, ivol=0, seed=41, nbrupdate=3)
    o, g = _pair(oracle_mod, gpu_lib, w)
    o.md_init()
    g.md_init()
    th_o = [o.md_step() for _ in range(12)]
    th_g = g.md_steps(12)
    for k in ("pe", "ke", "th"):
        a = np.array([t[k] for t in th_o])
        b = np.array([t[k] for t in th_g])
        assert np.max(np.abs(a - b)) < 1e-9 * np.max(np.abs(a)), k
    lo = o.linkcells()
    lg = g.linkcells(o.ncell)
    for a, b in zip(lo, lg):
        assert np.array_equal(a, b)


def test_kernel_variants_agree_and_autotune(oracle_mod, gpu_lib):
    """Every compiled variant of the pair passes gives the same FP64 forces
    (only the summation order may differ), and autotuning changes no state."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(10, sigma=0.05, temperature=600.0, ivol=0, seed=3)
    g = MoldySystem.from_workload(w)
    g.force()
    f0 = g.forces()
    for v in range(8):
        g.set_variants(v, 0, v)
        g.force()
        assert rel_norm_err(g.forces(), f0) < 1e-13
    s0 = g.get_state()
    tune = g.autotune(nreps=2)
    assert set(tune["chosen"]) == {"screen_density", "forces"}
    assert all(0 <= v < 8 for v in tune["chosen"].values())
    s1 = g.get_state()
    for k in ("x0", "x1", "x2", "b0", "b1"):
        assert np.array_equal(s0[k], s1[k]), k
    assert g.pair_count() > 13.0 * w.nm


def test_mixed_precision_accuracy(oracle_mod, gpu_lib):
    """Mixed path (FP32 distances, tables and pair forces; FP64 sums): force RMS
    error <= 1e-5 eV/A against FP64 on a 1200 K, 16,000-atom configuration;
    energy and stress errors are small and stated here."""
    from moldy_b200 import MoldySystem
    from moldy_b200 import units
    w = wl.make_workload(20, sigma=0.05, temperature=1200.0, ivol=0, seed=2)
    g64 = MoldySystem.from_workload(w, precision="fp64")
    gmx = MoldySystem.from_workload(w, precision="mixed")
    o64 = g64.force()
    omx = gmx.force()
    f64 = real_forces(g64.forces(), w.b0)
    fmx = real_forces(gmx.forces(), w.b0)
    rms = float(np.sqrt(np.mean((fmx - f64) ** 2)))
    assert rms <= 1e-5, rms
    assert abs(omx["pe"] - o64["pe"]) / w.nm < 1e-6            # eV/atom
    vol = o64["vol"]
    sig = lambda o: -(w.b0 @ (o["tp"]).T).T / vol * units.PRESS_TO_GPA
    assert np.max(np.abs(sig(omx) - sig(o64))) < 1e-4           # GPa


def test_md_hot_intermediate_list_rebuilds(oracle_mod, gpu_lib):
    """3000 K, 80 steps, no half-list rebuild: atoms move far enough that the
    intermediate list must be rebuilt from the displacement bound, and the
    trajectory still follows the oracle, which walks the whole half list."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(8, sigma=0.1, temperature=3000.0, ivol=1, seed=13, nbrupdate=200)
    o = oracle_mod.from_workload(w, uselookup=True, threads=1)
    g = MoldySystem.from_workload(w)
    o.md_init()
    g.md_init()
    th_o = [o.md_step() for _ in range(80)]
    th_g = g.md_steps(80)
    assert g.list_stats()["mid_builds"] >= 3
    a = np.array([t["pe"] for t in th_o])
    b = np.array([t["pe"] for t in th_g])
    assert np.max(np.abs(a - b)) < 1e-8 * np.max(np.abs(a))
    so, sg = o.get_state(), g.get_state()
    assert np.max(np.abs((sg["x0"] - so["x0"]) @ w.b0.T)) < 1e-7


def test_scalev_thermostat_matches_oracle(gpu_lib, oracle_mod):
    """mdloop with scalev (nose > 0) heating a 2000-atom NPT cell from 300 K
    towards 900 K: the GPU trajectory follows the oracle's (thermo within 1e-9
    relative over 60 steps), including snhv and the femtosecond timer."""
    from moldy_b200 import MoldySystem, units
    w = wl.make_workload(10, sigma=0.05, temperature=300.0, ivol=0, press_gpa=0.0, nbrupdate=20, seed=4)
    rqke = 1.5 * units.BK * 900.0 * (w.nm - 3)
    s = MoldySystem.from_workload(w)
    s.linkup()
    s.md_init()
    s.set_thermostat(5.0, rqke)
    g = s.md_steps(60)
    o = oracle_mod.from_workload(w, uselookup=True, threads=4)
    o.md_init()
    o.set_thermostat(5.0, rqke)
    r = [o.md_step() for _ in range(60)]
    for k in (0, 1, 2, 10, 30, 59):
        for key in ("ke", "pe", "te", "th", "temp"):
            assert abs(g[k][key] - r[k][key]) <= 1e-9 * abs(r[k][key]), (k, key, g[k][key], r[k][key])
    tg, to = s.thermostat(), o.thermostat()
    assert tg["snhv"] > 0.0          # kinetic energy below rqke: velocities scaled up
    assert abs(tg["snhv"] - to["snhv"]) <= 1e-9 * abs(to["snhv"])
    assert tg["thermotimer"] == to["thermotimer"]
    s.close()


def test_strainloops_ramp(gpu_lib):
    """The strain-loop temperature ramp: each loop raises rqke; the cell heats."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(10, sigma=0.05, temperature=300.0, ivol=0, press_gpa=0.0, nbrupdate=20, seed=6)
    s = MoldySystem.from_workload(w)
    s.linkup()
    s.md_init()
    recs, t_end = s.strainloops(4, 50, temprq=300.0, tempsp=200.0, nose=2.0)
    assert t_end == 1100.0 and len(recs) == 200
    assert recs[-1]["temprq"] == 1100.0
    assert np.mean([r["temp"] for r in recs[-20:]]) > np.mean([r["temp"] for r in recs[:20]]) + 100.0
    s.close()


def test_mid_skin_changes_no_result(gpu_lib):
    """The intermediate-list skin is a tuning knob: a thin skin (frequent
    device-decided rebuilds) and the default give the same trajectory."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(10, sigma=0.05, temperature=1500.0, ivol=0, seed=8, nbrupdate=50)
    runs = []
    for skin in (0.9, 0.25):
        s = MoldySystem.from_workload(w)
        s.set_mid_skin(skin)
        s.linkup()
        s.md_init()
        th = s.md_steps(80)
        runs.append((th, s.list_stats()["mid_builds"]))
        s.close()
    (a, na), (b, nb) = runs
    assert nb > na                       # the thin skin was rebuilt more often
    for k in (0, 40, 79):
        for key in ("pe", "ke", "th"):
            assert abs(a[k][key] - b[k][key]) <= 1e-10 * abs(a[k][key]), (k, key)


def test_outer_skin_changes_no_result(gpu_lib):
    """The outer-list skin is a tuning knob too: a thin outer skin (outer
    rebuilds decided on the device from the displacement since its build)
    and a thick one give the same trajectory."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(10, sigma=0.05, temperature=1500.0, ivol=0, seed=8, nbrupdate=200)
    runs = []
    for out in (2.0, 0.45):
        s = MoldySystem.from_workload(w)
        s.set_mid_skin(0.05)
        s.set_outer_skin(out)
        s.linkup()
        s.md_init()
        th = s.md_steps(80)
        runs.append((th, s.outer_builds(), s.list_stats()["mid_builds"]))
        s.close()
    (a, oa, ma), (b, ob, mb) = runs
    assert ob > oa >= 1 and ma > 3 and mb > 3
    for k in (0, 40, 79):
        for key in ("pe", "ke", "th"):
            assert abs(a[k][key] - b[k][key]) <= 1e-10 * abs(a[k][key]), (k, key)


def test_md_hot_outer_list_rebuilds(oracle_mod, gpu_lib):
    """3000 K with thin skins and no half-list rebuild in 60 steps: the outer
    list is rebuilt from its displacement bound several times, and the
    trajectory follows the oracle, which walks the whole half list."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(8, sigma=0.1, temperature=3000.0, ivol=1, seed=13, nbrupdate=200)
    o = oracle_mod.from_workload(w, uselookup=True, threads=1)
    g = MoldySystem.from_workload(w)
    g.set_mid_skin(0.05)
    g.set_outer_skin(0.45)
    o.md_init()
    g.md_init()
    th_o = [o.md_step() for _ in range(60)]
    th_g = g.md_steps(60)
    assert g.outer_builds() >= 3
    a = np.array([t["pe"] for t in th_o])
    b = np.array([t["pe"] for t in th_g])
    assert np.max(np.abs(a - b)) < 1e-8 * np.max(np.abs(a))
    so, sg = o.get_state(), g.get_state()
    assert np.max(np.abs((sg["x0"] - so["x0"]) @ w.b0.T)) < 1e-7


@pytest.mark.parametrize("ivol", [2, 5])
def test_partly_periodic_box_mixed_runs_fp64(oracle_mod, gpu_lib, ivol):
    """A box periodic in only some directions (ivol 2: x and y; ivol 5: z):
    the fixed-point minimum image of the mixed passes does not apply, so the
    mixed engine evaluates in FP64 and matches the FP64 engine bit for bit,
    and both match the oracle."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(8, sigma=0.05, temperature=600.0, ivol=ivol, seed=21)
    o = oracle_mod.from_workload(w, uselookup=True, threads=4)
    o.force()
    fo = o.force_out()
    res = []
    for prec in ("mixed", "fp64"):
        g = MoldySystem.from_workload(w, precision=prec)
        out = g.force()
        res.append((g.forces(), out))
        g.close()
    (fm, om), (fd, od) = res
    assert np.array_equal(fm, fd) and om["pe"] == od["pe"]
    assert rel_norm_err(fd, o.forces()) <= 1e-10
    assert abs(od["pe"] - fo["pe"]) <= 1e-10 * abs(fo["pe"])


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_md_bit_reproducible(gpu_lib, prec):
    """Two runs of the same MD (thin skins: several outer and intermediate
    list rebuilds) end in the same state bit for bit."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(8, sigma=0.1, temperature=2000.0, ivol=0, seed=17, nbrupdate=200)
    states = []
    for _ in range(2):
        s = MoldySystem.from_workload(w, precision=prec)
        s.set_mid_skin(0.05)
        s.set_outer_skin(0.45)
        s.linkup()
        s.md_init()
        s.md_steps(40)
        assert s.outer_builds() >= 2
        states.append((s.get_state(), s.forces()))
        s.close()
    (a, fa), (b, fb) = states
    for k in ("x0", "x1", "x2", "b0", "b1"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(fa, fb)


@pytest.mark.parametrize("prec,ivol", [("mixed", 0), ("fp64", 1)])
def test_md_steps_graph_replay_matches_launches(gpu_lib, prec, ivol):
    """md_steps replays a captured graph for its ordinary steps (the thermo
    record index kept on the device); with the library's profiling on it
    launches every kernel itself.  Both give the same state, forces and
    per-step thermo records bit for bit, over calls that cross half-list
    rebuilds and relinks (nbrupdate 25) and end on a last step of their own."""
    from moldy_b200 import MoldySystem
    w = wl.make_workload(8, sigma=0.1, temperature=1200.0, ivol=ivol, seed=31, nbrupdate=25)
    runs = []
    for prof in (True, False):
        s = MoldySystem.from_workload(w, precision=prec)
        s.set_profiling(prof)
        s.linkup()
        s.md_init()
        recs = s.md_steps(60, thermo=True) + s.md_steps(13, thermo=True)
        s.md_steps(9, thermo=False)
        recs += s.md_steps(30, thermo=True)
        runs.append((s.get_state(), s.forces(), recs))
        s.close()
    (a, fa, ra), (b, fb, rb) = runs
    for k in ("x0", "x1", "x2", "b0", "b1"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(fa, fb)
    assert len(ra) == len(rb) == 103
    for x, y in zip(ra, rb):
        assert x == y
