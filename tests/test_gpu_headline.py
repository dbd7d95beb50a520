"""Parity at the benchmarked size, through the C ABI against the CPU oracle.

* The 2,000,000-atom bcc Fe workload the benchmark times (100^3 bcc cells,
  a0 = 2.8665 A, sigma = 0.05 A, 1200 K, Parrinello-Rahman NPT, rnear = 6.3 A,
  45^3 = 91,125 link cells): the half list NLIST/NUMN is bit-exact; one FP64
  force call is within 1e-10 (norm-wise relative) in forces, rho, F'(rho),
  pe, the virial tp and fb; one mixed-precision call is within the accuracy
  gate against the oracle itself (real-force RMS <= 1e-5 eV/A, pe <= 1e-6
  eV/atom, stress <= 1e-4 GPa).
* The 2000-atom NVE workload (10^3 bcc cells, 300 K, dt 1 fs): 100 steps of
  the mixed path against 100 oracle steps, with the bounds stated below.

The oracle runs on every host thread here (OpenMP); its sums then change
order from run to run by rounding only, well inside the FP64 bound.
"""
import numpy as np
import pytest

from moldy_b200 import units
from moldy_b200 import workloads as wl
from tests.helpers import real_forces, rel_norm_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _stress_gpa(fo, b0):
    return -(b0 @ (fo["tp"]).T).T / fo["vol"] * units.PRESS_TO_GPA


@pytest.fixture(scope="module")
def headline(oracle_mod, gpu_lib):
    w = wl.config_large_npt()
    o = oracle_mod.from_workload(w, uselookup=True, threads=oracle_mod.max_threads())
    o.force()
    out = {"w": w, "fo": o.force_out(), "f": o.forces(), "dens": o.density()}
    out["nlist"], out["numn"] = o.nlist()
    o.close()
    return out


def test_headline_neighbour_list_exact(headline, gpu_lib):
    from moldy_b200 import MoldySystem
    h = headline
    w = h["w"]
    g = MoldySystem.from_workload(w, precision="fp64")
    g.force()
    nlg, nng = g.neighbour_list()
    g.close()
    assert w.nlc == (45, 45, 45)
    assert np.array_equal(nng, h["numn"])
    mask = np.arange(w.nnbrs, dtype=np.int32)[None, :] < h["numn"][:, None]
    assert np.array_equal(np.where(mask, h["nlist"], 0), nlg)
    assert int(h["numn"].sum()) > 40 * w.nm


def test_headline_force_fp64(headline, gpu_lib):
    from moldy_b200 import MoldySystem
    h = headline
    w = h["w"]
    g = MoldySystem.from_workload(w, precision="fp64")
    fg = g.force()
    assert rel_norm_err(g.forces(), h["f"]) < FP64_TOL
    dg = g.density()
    for k in ("rho", "dafrho"):
        assert rel_norm_err(dg[k], h["dens"][k]) < FP64_TOL, k
    assert abs(fg["pe"] - h["fo"]["pe"]) < FP64_TOL * abs(h["fo"]["pe"])
    for k in ("tp", "fb"):
        assert rel_norm_err(fg[k], h["fo"][k]) < FP64_TOL, k
    g.close()


def test_headline_force_mixed_vs_oracle(headline, gpu_lib):
    from moldy_b200 import MoldySystem
    h = headline
    w = h["w"]
    g = MoldySystem.from_workload(w, precision="mixed")
    fg = g.force()
    df = real_forces(g.forces(), w.b0) - real_forces(h["f"], w.b0)
    rms = float(np.sqrt(np.mean(np.sum(df * df, axis=1))))
    assert rms <= 1e-5, rms
    assert abs(fg["pe"] - h["fo"]["pe"]) / w.nm <= 1e-6
    assert np.max(np.abs(_stress_gpa(fg, w.b0) - _stress_gpa(h["fo"], w.b0))) <= 1e-4
    g.close()


def test_mixed_trajectory_2000_atoms_100_steps(oracle_mod, gpu_lib):
    """Mixed precision over 100 NVE steps against the FP64 oracle: the total
    energy per atom within 1e-6 eV at every step, pe and ke per atom within
    1e-5 eV, positions within 1e-4 A and velocities within 1e-4 A/fs at the
    end.  (The mixed forces differ from FP64 by about 2e-6 eV/A RMS.)"""
    from moldy_b200 import MoldySystem
    w = wl.config_small_nve()
    o = oracle_mod.from_workload(w, uselookup=True, threads=1)
    g = MoldySystem.from_workload(w, precision="mixed")
    o.md_init()
    g.md_init()
    th_o = [o.md_step() for _ in range(100)]
    th_g = g.md_steps(100)
    for k, tol in (("te", 1e-6), ("pe", 1e-5), ("ke", 1e-5)):
        a = np.array([t[k] for t in th_o])
        b = np.array([t[k] for t in th_g])
        assert np.max(np.abs(a - b)) / w.nm < tol, k
    so, sg = o.get_state(), g.get_state()
    assert np.max(np.abs((sg["x0"] - so["x0"]) @ w.b0.T)) < 1e-4
    dv = (sg["x1"] - so["x1"]) @ w.b0.T / w.meta["dt_fs"]
    assert np.max(np.abs(dv)) < 1e-4
    assert [t["ntc"] for t in th_g] == [int(t["ntc"]) for t in th_o]
