"""GPU analysis_m::rdf (src/analysis_m.F90:497-760) through the C ABI against
the oracle on the same state: histograms, atom counts, Ackland-Jones classes,
coordination and bond-angle counts are integers and must be identical; and
the all-pairs histogram of the GPU's own bcc-iron run against the
reference's shipped rdf.dat."""
import numpy as np
import pytest

from moldy_b200 import MoldyError, MoldySystem, analysis
from moldy_b200 import workloads as wl
from tests.helpers import bcc_iron_golden, bcc_iron_workload
from tests.test_rdf_oracle import check_against_rdf_golden

pytestmark = pytest.mark.gpu

MODE = {0: "list", 1: "all"}


def same_state(oracle_mod, w, steps=4):
    """Oracle MD steps, the same state on the GPU, and both half lists built
    at it (the lists agree entry by entry)."""
    o = oracle_mod.from_workload(w, uselookup=True, threads=4)
    if steps:
        o.linkup()
        o.md_init()
        for _ in range(steps):
            o.md_step()
    st = o.get_state()
    g = MoldySystem.from_workload(w)
    g.set_state(x0=st["x0"], b0=st["b0"])
    o.linkup()
    assert o.update_neighbourlist() == 0
    g.linkup()
    g.update_neighbourlist()
    return o, g


@pytest.mark.parametrize("mode", [0, 1])
def test_gpu_rdf_matches_oracle(oracle_mod, gpu_lib, mode):
    w = wl.make_workload(10, sigma=0.08, temperature=600.0, seed=3)
    o, g = same_state(oracle_mod, w)
    ho = o.rdf(300, 50, mode=mode)
    hg = analysis.rdf(g, 300, 50, MODE[mode])
    assert np.array_equal(ho["hist"], hg["hist"])
    assert np.array_equal(ho["natoms"], hg["natoms"]) and ho["nclose"] == hg["nclose"]
    assert hg["hist"].sum() > 20 * w.nm
    g.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_gpu_rdf_species_and_vacancies_match_oracle(oracle_mod, gpu_lib, mode):
    """Three species and every 37th site a vacancy (atomic number 0): the
    per-species-pair histograms and atom counts agree."""
    w = wl.make_workload(9, sigma=0.1, temperature=0.0, seed=8)
    w.atomic_number = w.atomic_number.copy()
    w.atomic_number[::37] = 0
    o, g = same_state(oracle_mod, w, steps=0)
    spec = np.random.default_rng(1).integers(0, 3, size=w.nm).astype(np.int32)
    ho = o.rdf(250, 50, mode=mode, spec=spec, nspec=3)
    hg = analysis.rdf(g, 250, 50, MODE[mode], species=spec, nspec=3)
    assert np.array_equal(ho["hist"], hg["hist"])
    assert np.array_equal(ho["natoms"], hg["natoms"])
    assert hg["natoms"].sum() == w.nm - len(range(0, w.nm, 37))
    g.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_gpu_ackland_jones_matches_oracle(oracle_mod, gpu_lib, mode):
    """Classes, coordination and the eight angle counts of every atom, with
    the radius the routine estimates from the histogram; a hot lattice gives
    a mixture of classes."""
    w = wl.make_workload(10, sigma=0.15, temperature=1500.0, seed=5)
    o, g = same_state(oracle_mod, w, steps=6)
    h = o.rdf(500, 50, mode=0)
    rn = oracle_mod.Oracle.rneighbour(h["hist"], h["natoms"], 50)
    assert np.array_equal(rn, analysis.rneighbour(h["hist"], h["natoms"], 50))
    ro = o.ackland_jones(rn, mode=mode)
    rg = analysis.ackland_jones(g, rn, MODE[mode])
    assert np.array_equal(ro["nn"], rg["nn"])
    assert np.array_equal(ro["chi"], rg["chi"])
    assert np.array_equal(ro["aj"], rg["aj"])
    assert len(np.unique(rg["aj"])) >= 2
    g.close()


def test_gpu_rdf_of_reference_bcc_iron_run(gpu_lib):
    """The GPU's FP64 bcc-iron run (IRON_CARBON tables, 10 NPT steps), then
    rdf(500, 50) over every pair, against the reference's shipped rdf.dat;
    the half-list form agrees with it below rnear = 6.4 A, and the warm
    lattice classifies as bcc with 14 neighbours (99 % of atoms at least)."""
    g = bcc_iron_golden()
    s = MoldySystem.from_workload(bcc_iron_workload(g))
    s.set_up_iron_carbon(nlookup=5000)
    s.linkup()
    s.md_init()
    s.md_steps(g["setup"]["steps"])
    res = analysis.rdf(s, 500, 50, "all")
    check_against_rdf_golden(res["hist"][:, 0, 0])
    s.linkup()
    s.update_neighbourlist()
    lst = analysis.rdf(s, 500, 50, "list")["hist"][:, 0, 0]
    assert np.array_equal(lst[:320], res["hist"][:320, 0, 0])
    rn = analysis.rneighbour(lst[:, None, None], [31250], 50)
    aj = analysis.ackland_jones(s, rn, "list")
    assert np.mean(aj["aj"] == 1) >= 0.99 and np.mean(aj["nn"] == 14) >= 0.99
    s.close()


def test_gpu_analyse_writes_the_reference_files(gpu_lib, tmp_path):
    w = wl.make_workload(8, sigma=0.05, temperature=300.0, seed=2)
    s = MoldySystem.from_workload(w)
    s.linkup()
    s.update_neighbourlist()
    out = analysis.analyse(s, 500, 50, directory=str(tmp_path))
    assert np.mean(out["aj"] == 1) >= 0.99
    rdf = open(tmp_path / "rdf.dat").read().splitlines()
    assert len(rdf) == 500 and rdf[0].split()[0] == "0.0200000"
    assert len(open(tmp_path / "prdf.dat").read().splitlines()) == 500
    aj = open(tmp_path / "aj_b1f2h3.dat").read().splitlines()
    assert len(aj) == w.nm + 1
    assert aj[1].split() == ["1", "26", str(out["aj"][0]), str(out["nn"][0])]
    s.close()


def test_gpu_rdf_rejects_bad_input(gpu_lib):
    w = wl.make_workload(4, sigma=0.0, temperature=0.0)
    s = MoldySystem.from_workload(w)
    s.linkup()
    s.update_neighbourlist()
    with pytest.raises(MoldyError):          # every box width must exceed 2 (maxbin+1)/bpa
        analysis.rdf(s, 500, 50, "all")
    with pytest.raises(MoldyError):
        analysis.rdf(s, 100, 50, "list", species=np.full(w.nm, 3), nspec=2)
    with pytest.raises(MoldyError):
        analysis.rdf(s, 100, 50, "list", species=np.zeros(w.nm), nspec=9)
    s.close()
