"""GPU parity of the batched supercells: one launch per pass over many
systems of uneven size, checked system by system against the oracle's
force() + energy_calc() and its VA14CD quench."""
import numpy as np
import pytest

from moldy_b200 import MoldyBatch
from moldy_b200 import workloads as wl
from tests.helpers import rel_norm_err

pytestmark = pytest.mark.gpu


def mixed_systems(sizes, seed=11, sigma=0.1):
    rng = np.random.default_rng(seed)
    return [wl.make_workload(n, sigma=sigma, temperature=0.0, ivol=1, seed=int(rng.integers(1 << 30)),
                             strain=wl.random_symmetric_strain(rng, 0.02)) for n in sizes]


def oracle_eval(oracle_mod, w):
    o = oracle_mod.from_workload(w, uselookup=True, threads=4)
    o.force()
    return o, o.energy_calc()


@pytest.mark.parametrize("tiles", [(8, 256), (4, 256), (32, 64), (16, 0)])
def test_batch_force_matches_oracle(gpu_lib, oracle_mod, tiles):
    """Forces, densities, per-atom energies, pe and the virial of every system
    within 1e-10 of the oracle; systems with 1-, 2-, 3- and more-cell grids, and
    tiles that spill past the staged capacity (staged 64 and 0)."""
    ws = mixed_systems([4, 5, 6, 7, 9, 4, 5])
    b = MoldyBatch.from_workloads(ws)
    b.set_tiles(*tiles)
    out = b.force()
    f = b.split(b.forces())
    ec, ef = (b.split(a) for a in b.energies())
    dens = b.density()
    rho = b.split(dens["rho"])
    for s, w in enumerate(ws):
        o, en = oracle_eval(oracle_mod, w)
        fo = o.force_out()
        assert rel_norm_err(f[s], o.forces()) <= 1e-10, s
        assert rel_norm_err(rho[s], o.density()["rho"]) <= 1e-10, s
        assert rel_norm_err(ec[s], en) <= 1e-10, s
        assert abs(out["pe_calc"][s] - en.sum()) <= 1e-10 * abs(en.sum())
        assert abs(out["pe"][s] - fo["pe"]) <= 1e-10 * abs(fo["pe"])
        assert rel_norm_err(out["tp"][s], fo["tp"]) <= 1e-10, s
        assert abs(out["vol"][s] - fo["vol"]) <= 1e-12 * fo["vol"]
    b.close()


@pytest.mark.parametrize("maxfn,skin", [(3, 0.3), (8, 0.3), (17, 0.3), (17, 0.0), (17, 1.0)])
def test_batch_quench_path_matches_oracle(gpu_lib, oracle_mod, maxfn, skin):
    """The first maxfn function values of VA14CD: with an unreachable force
    bound both the device state machine and the oracle stop at maxfn with
    iflag 1 at the best point so far; f agrees to 1e-11 and the positions to
    1e-9 A, so both took the same steps.  Skins 0 (a build at every
    evaluation), 0.3 and 1 A (lists kept through the line searches)."""
    ws = mixed_systems([4, 5, 6, 4, 7], seed=5)
    b = MoldyBatch.from_workloads(ws)
    b.set_skin(skin)
    q = b.quench(maxfn=maxfn, criterion=1, fmax=1e-12)
    xs = b.split(b.get_state())
    for s, w in enumerate(ws):
        o = oracle_mod.from_workload(w, uselookup=True, threads=4)
        r = o.quench(maxfn=maxfn, criterion=1, fmax=1e-12)
        assert q["iflag"][s] == 1 and r["iflag"] == 1
        assert q["nfev"][s] == r["nfev"] == maxfn
        assert q["iterations"][s] == r["iterations"]
        assert abs(q["f"][s] - r["f"]) <= 1e-11 * abs(r["f"]), (s, q["f"][s], r["f"])
        dx = (xs[s] - o.get_state()["x0"]) @ w.b0.T
        assert np.max(np.abs(dx)) <= 1e-9, s
    b.close()


def test_batch_quench_converges_like_oracle(gpu_lib, oracle_mod):
    """To max |F| <= 1e-4 eV/A: every system converges, its f within 1e-10 of
    the oracle's, and the oracle's energy at the GPU's final positions equals
    the GPU's f.  (Near the minimum the accept/reject decisions compare
    energies that differ in the last bits with the summation order, so the
    two may take different final steps.)"""
    ws = mixed_systems([4, 5, 6, 4, 5], seed=5)
    b = MoldyBatch.from_workloads(ws)
    q = b.quench(maxfn=2000, criterion=1, fmax=1e-4)
    xs = b.split(b.get_state())
    for s, w in enumerate(ws):
        r = oracle_mod.from_workload(w, uselookup=True, threads=4).quench(maxfn=2000, criterion=1, fmax=1e-4)
        assert q["iflag"][s] == 0 and r["iflag"] == 0
        assert q["fmax"][s] <= 1e-4
        assert abs(q["f"][s] - r["f"]) <= 1e-10 * abs(r["f"]), (s, q["f"][s], r["f"])
        w2 = w.copy()
        w2.x0 = xs[s]
        _, en2 = oracle_eval(oracle_mod, w2)
        assert abs(en2.sum() - q["f"][s]) <= 1e-12 * abs(q["f"][s])
    b.close()


def test_batch_quench_reference_criterion(gpu_lib, oracle_mod):
    """The reference's acceptance (sum of squared gradient <= 5e-7 nm): a
    system either meets it (iflag 0) or ends, as the oracle's VA14CD also does
    for some systems, with the conjugate-gradient error return (iflag 2) at
    the precision floor; either way f is the oracle's within 1e-9."""
    ws = mixed_systems([4, 5, 6, 4, 5], seed=5)
    b = MoldyBatch.from_workloads(ws)
    q = b.quench(maxfn=2000, criterion=0)
    for s, w in enumerate(ws):
        r = oracle_mod.from_workload(w, uselookup=True, threads=4).quench(maxfn=2000, criterion=0)
        assert q["iflag"][s] in (0, 2)
        if q["iflag"][s] == 0:
            assert q["gsumsq"][s] <= 5e-7 * w.nm
        assert abs(q["f"][s] - r["f"]) <= 1e-9 * abs(r["f"]), (s, q["f"][s], r["f"])
    b.close()


def test_batch_many_systems_converge(gpu_lib, oracle_mod):
    """64 systems of 128 to 2000 atoms quenched towards max |F| <= 1e-4 eV/A.
    derivs differentiates the tabulated forces but takes the energy from
    energy_calc's exact pair function, so f and g disagree at about 1e-4 eV/A
    and VA14CD ends some systems with its conjugate-gradient error return
    (iflag 2) just above the bound, as the oracle does for the same systems.
    Every other system meets the bound; a sample matches the oracle's f."""
    ws = wl.config_batch(nsys=64, seed=9, n_range=(4, 10))
    b = MoldyBatch.from_workloads(ws)
    e0 = b.force()["pe_calc"]
    q = b.quench(maxfn=3000, criterion=1, fmax=1e-4)
    assert np.all((q["iflag"] == 0) | (q["iflag"] == 2))
    assert np.all(q["fmax"][q["iflag"] == 0] <= 1e-4)
    assert np.all(q["fmax"] <= 5e-4)
    assert np.mean(q["iflag"] == 0) >= 0.9
    assert np.all(q["f"] < e0)
    for s in [0, 17, 41] + list(np.nonzero(q["iflag"] == 2)[0][:2]):
        r = oracle_mod.from_workload(ws[s], uselookup=True, threads=4).quench(maxfn=3000, criterion=1, fmax=1e-4)
        assert abs(q["f"][s] - r["f"]) <= 1e-9 * abs(r["f"])
        if q["iflag"][s] == 2:
            assert r["iflag"] == 2
    b.close()


def test_batch_rejects_narrow_box(gpu_lib):
    from moldy_b200 import MoldyError
    w = wl.make_workload(2, sigma=0.0, temperature=0.0, ivol=1)
    with pytest.raises(MoldyError):
        MoldyBatch.from_workloads([w])


def test_batch_list_kept_until_half_skin(gpu_lib, oracle_mod):
    """A system's list is kept while its atoms stay within half the skin of
    their positions at the last build, and rebuilt (that system alone) once
    one atom moves farther; the results match the oracle at every step."""
    ws = mixed_systems([4, 5, 6, 4], seed=21)
    b = MoldyBatch.from_workloads(ws)
    b.set_skin(0.4)
    b.force()
    assert b.list_stats() == {"builds": 4, "evaluations": 4}
    rng = np.random.default_rng(4)
    x0 = [w.x0.copy() for w in ws]

    def move(s, cart):
        return np.linalg.solve(ws[s].b0, cart.T).T

    # every atom of every system moves by less than 0.15 A: no build
    xs = [x0[s] + move(s, rng.uniform(-0.08, 0.08, size=(ws[s].nm, 3))) for s in range(4)]
    b.set_state(np.concatenate(xs))
    b.force()
    assert b.list_stats() == {"builds": 4, "evaluations": 8}
    f = b.split(b.forces())
    for s, w in enumerate(ws):
        w2 = w.copy()
        w2.x0 = xs[s]
        o, _ = oracle_eval(oracle_mod, w2)
        assert rel_norm_err(f[s], o.forces()) <= 1e-10, s
    # one atom of system 2 moves 0.25 A from its built position: that system rebuilds
    xs[2] = xs[2].copy()
    xs[2][7] = x0[2][7] + move(2, np.array([[0.25, 0.0, 0.0]]))[0]
    b.set_state(np.concatenate(xs))
    out = b.force()
    assert b.list_stats() == {"builds": 5, "evaluations": 12}
    f = b.split(b.forces())
    for s, w in enumerate(ws):
        w2 = w.copy()
        w2.x0 = xs[s]
        o, en = oracle_eval(oracle_mod, w2)
        assert rel_norm_err(f[s], o.forces()) <= 1e-10, s
        assert abs(out["pe_calc"][s] - en.sum()) <= 1e-10 * abs(en.sum())
    # a new box rebuilds every list
    b.set_state(b0=[w.b0 for w in ws])
    b.force()
    assert b.list_stats()["builds"] == 9
    b.close()


def test_batch_interleaved_copies(gpu_lib):
    """set_positions / forces_xyz_into carry the same numbers as the
    per-component calls."""
    ws = mixed_systems([4, 5], seed=2)
    b = MoldyBatch.from_workloads(ws)
    b.force()
    f1 = b.forces()
    x = np.ascontiguousarray(np.concatenate([w.x0 for w in ws]))
    x[3] += 1e-3
    b.set_positions(x)
    assert np.array_equal(b.get_state(), x)
    b.force()
    f2 = np.empty_like(f1)
    b.forces_xyz_into(f2)
    assert np.array_equal(f2, b.forces())
    assert not np.array_equal(f1, f2)
    with pytest.raises(ValueError):
        b.set_positions(x[:, :2])
    out = b.force()
    raw = np.zeros(13 * b.nsys)
    b.force_into(raw)
    raw = raw.reshape(b.nsys, 13)
    assert np.array_equal(raw[:, 0], out["pe_calc"]) and np.array_equal(raw[:, 1], out["pe"])
    assert np.array_equal(raw[:, 4:13].reshape(b.nsys, 3, 3).transpose(0, 2, 1), out["tp"])
    b.close()


def test_batch_gather_bit_identical(gpu_lib):
    """Row entries gathered 1, 2 or 4 at a time are summed in the same order:
    forces, energies, densities and the per-system virial are bit-identical."""
    ws = mixed_systems([4, 6, 5], seed=8)
    b = MoldyBatch.from_workloads(ws)
    res = []
    for g in (1, 2, 4):
        b.set_gather(g)
        out = b.force()
        res.append((b.forces(), *b.energies(), b.density()["rho"], out["tp"], out["pe_calc"]))
    for other in res[1:]:
        for x, y in zip(res[0], other):
            assert np.array_equal(x, y)
    with pytest.raises(Exception):
        b.set_gather(3)
    b.close()


def real_force_rms(ws, fa, fb):
    d = np.concatenate([(x - y) @ w.b0.T for w, x, y in zip(ws, fa, fb)])
    return float(np.sqrt(np.mean(np.sum(d * d, axis=1))))


def test_batch_mixed_accuracy(gpu_lib, oracle_mod):
    """Mixed precision (FP32 separations, tables and pair forces, FP64 sums)
    against the oracle, at the accuracy gate of the mixed path: real-force RMS
    error <= 1e-5 eV/A, both energies within 1e-6 eV/atom, rho within 1e-6
    and the virial within 1e-5 relative.  (An FP32 distance carries about
    2e-7 A of rounding, which the tables pass on to rho and F(rho).)"""
    ws = mixed_systems([4, 5, 6, 7, 9], seed=13)
    b = MoldyBatch.from_workloads(ws)
    b.set_precision("mixed")
    for g in (1, 4):
        b.set_gather(g)
        out = b.force()
        f = b.split(b.forces())
        rho = b.split(b.density()["rho"])
        fo_all = []
        for s, w in enumerate(ws):
            o, en = oracle_eval(oracle_mod, w)
            fo = o.force_out()
            fo_all.append(o.forces())
            assert rel_norm_err(rho[s], o.density()["rho"]) <= 1e-6, s
            assert abs(out["pe_calc"][s] - en.sum()) <= 1e-6 * w.nm, s
            assert abs(out["pe"][s] - fo["pe"]) <= 1e-6 * w.nm, s
            assert rel_norm_err(out["tp"][s], fo["tp"]) <= 1e-5, s
        assert real_force_rms(ws, f, fo_all) <= 1e-5
    b.close()


def test_batch_quench_stays_fp64(gpu_lib):
    """The quench evaluates in FP64 whatever force() uses: with mixed
    precision set, its results are bit-identical to the FP64 quench's."""
    ws = mixed_systems([4, 5, 6], seed=5)
    out = []
    for p in ("fp64", "mixed"):
        b = MoldyBatch.from_workloads(ws)
        b.set_precision(p)
        q = b.quench(maxfn=40, criterion=1, fmax=1e-4)
        out.append((q["f"], q["nfev"], b.get_state()))
        b.close()
    for x, y in zip(*out):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_autotune_and_energy_calc_switch(gpu_lib, precision):
    """moldy_gpu_batch_autotune picks a lanes/gather pair from its sets and
    changes no result: forces, pe and the virial after it equal, bit for bit,
    those of the default tiles.  With energy_calc switched off the energy_calc
    sums read zero and everything else is again bit-identical."""
    ws = mixed_systems([4, 5, 6, 7, 9, 4, 5], seed=21)
    b = MoldyBatch.from_workloads(ws)
    b.set_precision(precision)
    b.set_persistent(False)     # the per-pass launches throughout (the persistent one has its own tests)
    out0 = b.force()
    f0 = b.forces()
    tune = b.autotune(nreps=2)
    assert tune["chosen"]["lanes"] in (4, 8, 16, 32) and tune["chosen"]["gather"] in (1, 2, 4)
    assert all(t > 0 for t in tune["lanes_ms"].values()) and all(t > 0 for t in tune["gather_ms"].values())
    out1 = b.force()
    assert np.array_equal(b.forces(), f0)
    for k in ("pe_calc", "pe", "tp", "vol"):
        assert np.array_equal(out1[k], out0[k]), k
    b.set_energy_calc(False)
    out2 = b.force()
    assert np.array_equal(b.forces(), f0)
    assert np.all(out2["pe_calc"] == 0.0) and np.all(b.energies()[0] == 0.0)
    for k in ("pe", "tp", "vol"):
        assert np.array_equal(out2[k], out0[k]), k
    b.set_energy_calc(True)
    assert np.array_equal(b.force()["pe_calc"], out0["pe_calc"])
    kt = b.kernel_times(rebuild=True)
    assert set(kt) == {"prepare", "tile_screen", "density", "forces"} and all(v > 0 for v in kt.values())
    assert np.array_equal(b.forces(), f0)
    assert 10 * b.ntot < b.row_entries() < 40 * b.ntot
    b.close()


def test_batch_persistent_evaluation(gpu_lib, oracle_mod):
    """The persistent launch (mixed, energy_calc off): every system against the
    oracle at the mixed path's accuracy gate, and against the per-pass mixed
    launches, for 1, 2 and 4 lanes per atom; two evaluations bit for bit the
    same; lists rebuilt inside the launch (after a new skin) give the same
    results as the per-pass path's rebuild; a massless atom, FP64 or
    energy_calc switch it off."""
    ws = mixed_systems([4, 5, 6, 7, 9, 4, 5, 8], seed=23)
    b = MoldyBatch.from_workloads(ws)
    b.set_precision("mixed")
    b.set_energy_calc(False)
    assert b.persistent_applies()
    ref = []
    for w in ws:
        o, _ = oracle_eval(oracle_mod, w)
        ref.append((o.forces(), o.density()["rho"], o.force_out()))
    b.set_persistent(False)
    outp = b.force()
    fp_ = b.forces()
    b.set_persistent(True)
    for lanes in (1, 2, 4):
        b.set_atom_lanes(lanes)
        l0 = b.launches()
        out = b.force()
        assert b.launches() - l0 == 2          # the activity flags and the evaluation
        f = b.forces()
        rho = b.split(b.density()["rho"])
        for s, w in enumerate(ws):
            fo, rho_o, fout = ref[s]
            assert rel_norm_err(rho[s], rho_o) <= 1e-6, (lanes, s)
            assert abs(out["pe"][s] - fout["pe"]) <= 1e-6 * w.nm, (lanes, s)
            assert rel_norm_err(out["tp"][s], fout["tp"]) <= 1e-5, (lanes, s)
            assert out["vol"][s] == outp["vol"][s]
        assert real_force_rms(ws, b.split(f), [r[0] for r in ref]) <= 1e-5, lanes
        assert rel_norm_err(f, fp_) <= 1e-6, lanes
        assert np.all(out["pe_calc"] == 0.0)
        out_again = b.force()
        assert np.array_equal(b.forces(), f)
        for k in ("pe", "tp", "fmax"):
            assert np.array_equal(out_again[k], out[k]), k
    # rebuilds inside the launch: a new skin marks every list stale
    b.set_atom_lanes(2)
    st0 = b.list_stats()
    b.set_skin(0.25)
    b.force()
    assert b.list_stats()["builds"] - st0["builds"] == len(ws)
    f_rb = b.forces()
    e_rb = b.energies()[1]
    rows_rb = b.row_entries()
    b.set_persistent(False)
    b.set_skin(0.25)
    b.force()
    assert b.row_entries() == rows_rb
    assert rel_norm_err(f_rb, b.forces()) <= 1e-6
    assert rel_norm_err(e_rb, b.energies()[1]) <= 1e-6
    b.set_persistent(True)
    t = b.eval_times()
    assert t["current"] > 0 and t["rebuilt"] > 0
    tune = b.autotune(nreps=1)
    assert tune["chosen"]["atom_lanes"] in (1, 2, 4) and set(tune["atom_lanes_ms"]) == {1, 2, 4}
    b.set_energy_calc(True)
    assert not b.persistent_applies()
    b.set_energy_calc(False)
    b.set_precision("fp64")
    assert not b.persistent_applies()
    b.set_precision("mixed")
    m = np.full(b.ntot, 55.845)
    m[3] = 0.0
    b.set_state(mass=m)
    assert not b.persistent_applies()
    b.close()
