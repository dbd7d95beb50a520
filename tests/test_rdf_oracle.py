"""The oracle's restatement of analysis_m::rdf (src/analysis_m.F90:497-760)
pinned against the reference's shipped bcc-iron rdf.dat, checked for self-
consistency and on perfect lattices; the product's host-side radius estimate
and file writers against the oracle and the reference's formats."""
import json
import os

import numpy as np

from moldy_b200 import analysis
from moldy_b200 import workloads as wl
from tests.helpers import bcc_iron_golden, bcc_iron_workload
from tests.test_golden_bcc_iron import run_oracle


def rdf_golden():
    return json.load(open(os.path.join(os.path.dirname(__file__), "golden", "bcc_iron_rdf.json")))


def check_against_rdf_golden(counts):
    """counts[1..500] against the shipped histogram.  Its run came from an
    older version of the code whose final positions differ from the
    reproduced run by about 1e-7 A, which moves a few pairs in 1e5 across a
    bin edge: the pair total must be exact, the cumulative histogram within
    32 pairs everywhere and the summed bin differences within 1e-4 of all
    pairs."""
    g = np.array(rdf_golden()["counts"], dtype=np.int64)
    c = np.asarray(counts, dtype=np.int64)[1:]
    assert c.sum() == g.sum() == 5277662
    assert np.max(np.abs(np.cumsum(c) - np.cumsum(g))) <= 32
    assert np.abs(c - g).sum() <= 1e-4 * g.sum()
    assert np.all((c == 0) == (g == 0))


def test_oracle_rdf_matches_shipped_bcc_iron_rdf(oracle_mod):
    """rdf(500, 50) after the 10-step bcc-iron run: every pair with
    int(r * 50) <= 500, as the older all-pairs routine that wrote the file."""
    g = bcc_iron_golden()
    o, _ = run_oracle(oracle_mod, bcc_iron_workload(g), g["setup"]["steps"])
    res = o.rdf(500, 50, mode=1)
    assert res["hist"][0].sum() == 0 and res["nclose"] == 0
    check_against_rdf_golden(res["hist"][:, 0, 0])
    assert res["natoms"][0] == 31250


def small_oracle(oracle_mod, n=8, steps=5, seed=2):
    w = wl.make_workload(n, sigma=0.05, temperature=300.0, ivol=1, seed=seed)
    o = oracle_mod.from_workload(w, uselookup=True, threads=oracle_mod.max_threads())
    o.linkup()
    o.md_init()
    for _ in range(steps):
        o.md_step()
    o.linkup()
    o.update_neighbourlist()
    return w, o


def test_oracle_rdf_list_equals_all_pairs_on_a_fresh_list(oracle_mod):
    """With the half list just built (rnear 6.3 A), the list-mode histogram
    (rsq <= (300/50)^2) equals the all-pairs one below 6 A; the all-pairs
    form also keeps r in [6, 6.02) in bin 300."""
    w, o = small_oracle(oracle_mod)
    a = o.rdf(300, 50, mode=0)["hist"][:, 0, 0]
    b = o.rdf(300, 50, mode=1)["hist"][:, 0, 0]
    assert np.array_equal(a[:300], b[:300])
    assert a[300] <= b[300]
    assert a.sum() > 20 * w.nm


def lattice(kind, reps):
    """Perfect lattice: fractional positions (nm, 3) and box (columns are box
    vectors)."""
    if kind == "bcc":
        basis, cell = np.array([[0, 0, 0], [0.5, 0.5, 0.5]]), np.diag([2.8665] * 3)
    elif kind == "fcc":
        basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
        cell = np.diag([3.6] * 3)
    else:   # hcp, ideal c/a, orthorhombic cell of 4 atoms
        a = 2.5
        basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 1 / 6, 0.5], [0, 2 / 3, 0.5]])
        cell = np.diag([a, a * np.sqrt(3), a * np.sqrt(8 / 3)])
    r = np.array(reps)
    g = np.stack(np.meshgrid(*[np.arange(k) for k in r], indexing="ij"), -1).reshape(-1, 3)
    x = ((g[:, None, :] + basis[None, :, :]) / r).reshape(-1, 3)
    return x, cell @ np.diag(r)


def oracle_from_positions(oracle_mod, x, b0, ivol=1):
    nm = len(x)
    o = oracle_mod.Oracle(nm, nnbrs=150, ivol=ivol, ntcm=100)
    z = np.zeros((nm, 3))
    o.set_state(x, z, z, b0, np.zeros((3, 3)), np.zeros((3, 3)), np.full(nm, 26), np.full(nm, 55.845),
                np.full(nm, 1e-4))
    return o


def test_oracle_ackland_jones_perfect_lattices(oracle_mod):
    """bcc: class 1 with 14 neighbours; fcc: class 2 with 12; hcp: class 3
    with 12; every atom of a perfect lattice has the same angle counts.  (The
    reference's ibcc/ifcc/ihcp templates feed only crysdiff, whose result is
    unused, and do not follow its own ctheta windows: a first-to-second-shell
    bcc angle, cos = -0.577, falls in the band the routine skips.)"""
    expect = {"bcc": (1, 14, [7, 0, 0, 0, 12, 0, 36, 0]), "fcc": (2, 12, None), "hcp": (3, 12, None)}
    reps = {"bcc": (5, 5, 5), "fcc": (4, 4, 4), "hcp": (5, 3, 3)}
    for kind, (cls, nn, chi) in expect.items():
        x, b0 = lattice(kind, reps[kind])
        o = oracle_from_positions(oracle_mod, x, b0)
        h = o.rdf(300, 50, mode=1)
        rn = oracle_mod.Oracle.rneighbour(h["hist"], h["natoms"], 50)
        r = o.ackland_jones(rn, mode=1)
        assert np.all(r["aj"] == cls), (kind, np.bincount(r["aj"]))
        assert np.all(r["nn"] == nn), kind
        assert np.all(r["chi"] == r["chi"][0]), kind
        if chi is not None:
            assert np.array_equal(r["chi"][0], chi), (kind, r["chi"][0])


def test_host_rneighbour_matches_oracle(oracle_mod):
    """The product's host-side radius estimate equals the oracle's, species
    pairs and the carried-over value included."""
    rng = np.random.default_rng(5)
    for ns in (1, 2, 3):
        hist = rng.integers(0, 40, size=(301, ns, ns)).astype(np.int64)
        natoms = rng.integers(0, 500, size=ns).astype(np.int64)
        natoms[0] = 0 if ns == 3 else natoms[0]
        a = analysis.rneighbour(hist, natoms, 50)
        b = oracle_mod.Oracle.rneighbour(hist, natoms, 50)
        assert np.array_equal(a, b)


def test_rdf_file_formats(tmp_path):
    """rdf.dat '(F13.7,F18.7)', prdf.dat '(F13.7,F18.7,2I4)' and the
    list-directed aj_b1f2h3.dat, with single-precision radii."""
    hist = np.zeros((4, 1, 1), dtype=np.int64)
    hist[2, 0, 0] = 7
    analysis.write_rdf(tmp_path / "rdf.dat", hist, 50)
    lines = open(tmp_path / "rdf.dat").read().splitlines()
    assert len(lines) == 3 and all(len(l) == 31 for l in lines)
    r = np.float32(2) / np.float32(50)
    assert lines[1] == f"{float(r):13.7f}{float(np.float32(7) / (r * r)):18.7f}"
    assert lines[1].split()[0] == "0.0400000"
    analysis.write_prdf(tmp_path / "prdf.dat", hist, 50)
    assert open(tmp_path / "prdf.dat").read().splitlines()[1].endswith("   1   1")
    analysis.write_aj(tmp_path / "aj.dat", np.array([1, 0]), np.array([14, 9]), np.array([26, 26]))
    aj = open(tmp_path / "aj.dat").read().splitlines()
    assert aj[1] == "           1          26           1          14"
