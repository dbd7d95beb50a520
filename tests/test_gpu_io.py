"""The device engine with the on-disk formats (src/io_m.F90:73-379,
src/moldin.F90:983-1070): the GPU's FP64 bcc-iron run against the
reference's full-precision checkpoint, a device state carried through the
checkpoint format into a fresh engine, and a system.in read into the engine
against the oracle."""
import numpy as np
import pytest

from moldy_b200 import MoldySystem, io
from moldy_b200 import workloads as wl
from tests.helpers import bcc_iron_golden, bcc_iron_workload, rel_norm_err
from tests.test_io import check_state_against_checkpoint, io_golden

pytestmark = pytest.mark.gpu


def test_gpu_final_state_equals_reference_checkpoint(gpu_lib):
    """The GPU's FP64 10-step bcc-iron run against the reference's checkpoint:
    its sums run in another order than the reference's, so the bounds are
    looser than the oracle's (positions 1e-13, velocities and accelerations
    1e-9 relative, box 1e-15)."""
    g = bcc_iron_golden()
    s = MoldySystem.from_workload(bcc_iron_workload(g))
    s.set_up_iron_carbon(nlookup=5000)
    s.linkup()
    s.md_init()
    s.md_steps(g["setup"]["steps"])
    check_state_against_checkpoint(s.get_state(), 1e-13, 1e-9, 1e-15)
    s.close()


def test_gpu_state_through_checkpoint(gpu_lib, tmp_path):
    """A state after three NPT steps, written as a checkpoint with the
    reference's compiler-layout records and read into a fresh engine, is the
    same state bit for bit and gives the same forces and stress."""
    g = io_golden()["checkpoint"]
    w = wl.make_workload(8, sigma=0.05, temperature=600.0, ivol=0, seed=3)
    a = MoldySystem.from_workload(w)
    a.linkup()
    a.md_init()
    a.md_steps(3)
    st = a.get_state()
    template = io.Checkpoint(bytes.fromhex(g["simparam_hex"]), [], [], np.zeros(0), np.zeros(0), np.zeros(0),
                             np.array(g["ispec"]), bytes.fromhex(g["thmsums_hex"]))
    ck = io.checkpoint_from_state(st, template, w.atomic_number, w.atomic_mass, np.ones(w.nm, dtype=int))
    io.write_checkpoint(tmp_path / "chkp.dat", ck)
    back = io.read_checkpoint(tmp_path / "chkp.dat")
    b = MoldySystem.from_workload(w)
    b.set_state(**io.state_arrays(back))
    sb = b.get_state()
    for k in ("x0", "x1", "x2", "b0", "b1", "b2"):
        assert np.array_equal(st[k], sb[k]), k
    fa, fb = a.force(), b.force()
    assert rel_norm_err(b.forces(), a.forces()) <= 1e-12
    assert rel_norm_err(fb["tp"], fa["tp"]) <= 1e-12 and abs(fb["pe"] - fa["pe"]) <= 1e-12 * abs(fa["pe"])
    a.close()
    b.close()


def test_gpu_runs_a_system_in(oracle_mod, gpu_lib):
    """The reference's thermal system.in (2,000 atoms, offset basis, unequal
    box edges) read on the host and evaluated on the device: forces, pe and
    virial within 1e-10 of the oracle's on the same state."""
    s = io.read_system_in(io_golden()["system_in"]["thermal"])
    w = wl.make_workload(10, sigma=0.0, temperature=0.0, ivol=1)
    w.x0, w.b0 = s.x0, s.b0
    w.atomic_number, w.atomic_mass = s.atomic_number, s.atomic_mass
    w.del2 = w.deltat ** 2 / (2.0 * w.atomic_mass)
    o = oracle_mod.from_workload(w, uselookup=True, threads=4)
    o.force()
    fo = o.force_out()
    g = MoldySystem.from_workload(w)
    fg = g.force()
    assert rel_norm_err(g.forces(), o.forces()) <= 1e-10
    assert abs(fg["pe"] - fo["pe"]) <= 1e-10 * abs(fo["pe"])
    assert rel_norm_err(fg["tp"], fo["tp"]) <= 1e-10
    g.close()
