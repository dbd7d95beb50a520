"""The oracle against the reference's own shipped golden run
(tests/reference/bcc_iron of the reference: 31,250-atom bcc iron, IRON_CARBON
Fe-Fe potential in lookup mode, setvel at 600 K, 10 Parrinello-Rahman NPT
velocity-Verlet steps at 0.1 GPa).  Every printed digit of the step-10
thermodynamics and stress, the full-precision final box, and a sample of the
final positions and per-atom energies must agree.  The fixture is
tests/golden/bcc_iron_step10.json (written by make_bcc_iron_golden.py)."""
import numpy as np

from moldy_b200 import units
from tests.helpers import bcc_iron_golden, bcc_iron_workload, check_against_bcc_iron_golden


def run_oracle(oracle_mod, w, steps):
    o = oracle_mod.from_workload(w, uselookup=True, threads=oracle_mod.max_threads())
    o.set_iron_carbon()
    o.set_lookup(True, 5000)
    o.set_nlc(*w.nlc)
    o.linkup()
    o.md_init()
    r = None
    for _ in range(steps):
        r = o.md_step()
    return o, r


def test_iron_carbon_functions_match_shipped_table(oracle_mod):
    """The restated IRON_CARBON Fe-Fe V, V', phi, phi' against the reference's
    tabulation potential.55 (4 printed digits; the r column is itself printed
    to 4 digits, so r is taken from a fitted uniform grid and the tolerance
    adds |f'(r)| times the grid uncertainty)."""
    g = bcc_iron_golden()
    d = np.array([[float(v) for v in row] for row in g["potential55"]])
    o = oracle_mod.Oracle(16, nnbrs=8, ivol=1, ntcm=1)
    o.set_iron_carbon()
    k = np.arange(len(d))
    b, a = np.polyfit(k, d[:, 0], 1)
    r = a + b * k
    for j in range(4):
        v = np.array([o.src(j, x) for x in r])
        vp = np.array([(o.src(j, x + 1e-7) - o.src(j, x - 1e-7)) / 2e-7 for x in r])
        ref = d[:, j + 1]
        ulp = np.where(ref != 0, 10.0 ** (np.floor(np.log10(np.abs(np.where(ref != 0, ref, 1.0)))) - 3), 0.0)
        tol = 0.5 * ulp + np.abs(vp) * 3e-5 + 1e-6
        assert np.all(np.abs(v - ref) <= tol), (j, np.max(np.abs(v - ref) - tol))


def test_oracle_reproduces_reference_bcc_iron_run(oracle_mod):
    g = bcc_iron_golden()
    w = bcc_iron_workload(g)
    o, r = run_oracle(oracle_mod, w, g["setup"]["steps"])
    fo = o.force_out()
    st = o.get_state()
    b0 = st["b0"]
    stress = -(fo["tp"] @ b0.T) / fo["vol"] * units.PRESS_TO_GPA
    check_against_bcc_iron_golden(g, r, stress, b0, st["x0"], o.energy_calc())


def test_host_iron_carbon_tables_match_oracle(oracle_mod):
    """The product's table builder (moldy_ic_build_tables) equals the oracle's
    tables bit for bit."""
    from moldy_b200 import _lib, build
    build.build()
    L = _lib.load()
    t = [np.zeros(5001) for _ in range(6)]
    _lib.check(L.moldy_ic_build_tables(5000, *[a.ctypes.data_as(_lib.D) for a in t]))
    o = oracle_mod.Oracle(16, nnbrs=8, ivol=1, ntcm=1)
    o.set_iron_carbon()
    o.set_lookup(True, 5000)
    ref = o.tables()
    for k, name in enumerate(["vee", "dvee", "phi", "dphi", "emb", "demb"]):
        a, b = t[k], ref[name]
        same = (a == b) | (np.isnan(a) & np.isnan(b))
        assert np.all(same), (name, np.nonzero(~same)[0][:5])
