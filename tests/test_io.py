"""system.in, system.out and the unformatted checkpoint (src/io_m.F90:73-379,
src/moldin.F90:983-1070) against the reference's shipped test files (fixture
tests/golden/bcc_iron_io.json, written by make_bcc_iron_io_golden.py): the
product's readers and writers, and the oracle's final bcc-iron state against
the reference's full-precision checkpoint of the same run."""
import json
import os

import numpy as np
import pytest

from moldy_b200 import io
from moldy_b200 import workloads as wl
from tests.helpers import bcc_iron_golden, bcc_iron_workload
from tests.test_golden_bcc_iron import run_oracle


def io_golden():
    return json.load(open(os.path.join(os.path.dirname(__file__), "golden", "bcc_iron_io.json")))


def golden_checkpoint_sample(g):
    ck = g["checkpoint"]
    idx = np.array([int(k) for k in ck["atoms"]])
    x = [np.array([[float.fromhex(v) for v in ck["atoms"][str(i)]["x"][k]] for i in idx]) for k in range(4)]
    b = [np.array([float.fromhex(v) for v in box]).reshape(3, 3, order="F") for box in ck["boxes"]]
    return idx, x, b


def check_state_against_checkpoint(state, x_tol, v_tol, b_tol):
    """The final state of the reference's bcc-iron run (its chkp_out.dat):
    fractional positions within x_tol, velocities and accelerations within
    v_tol of their largest magnitude, the box within b_tol and the box
    velocity and acceleration within v_tol relative; the jolt terms are 0."""
    idx, x, b = golden_checkpoint_sample(io_golden())
    assert np.max(np.abs(state["x0"][idx] - x[0])) <= x_tol
    for k, name in ((1, "x1"), (2, "x2")):
        assert np.max(np.abs(state[name][idx] - x[k])) <= v_tol * np.abs(x[k]).max(), name
    assert np.max(np.abs(state["b0"] - b[0])) <= b_tol
    for k, name in ((1, "b1"), (2, "b2")):
        assert np.max(np.abs(state[name] - b[k])) <= v_tol * np.abs(b[k]).max(), name
    assert not np.any(x[3]) and not np.any(b[3])


def test_oracle_final_state_equals_reference_checkpoint(oracle_mod):
    """The oracle's 10-step bcc-iron run ends where the reference's did, to
    the last bits: positions 1e-19, velocities and accelerations 1e-15
    relative, box 1e-21 (measured); bounds 100-1000 times larger."""
    g = bcc_iron_golden()
    o, _ = run_oracle(oracle_mod, bcc_iron_workload(g), g["setup"]["steps"])
    check_state_against_checkpoint(o.get_state(), 1e-16, 1e-12, 1e-18)


def test_checkpoint_written_like_the_reference(oracle_mod, tmp_path):
    """A checkpoint of the oracle's final state with the reference's
    compiler-layout records has the reference file's record layout, reads
    back bit for bit, and its sampled atoms equal the reference's."""
    g = io_golden()
    ckg = g["checkpoint"]
    gb = bcc_iron_golden()
    o, _ = run_oracle(oracle_mod, bcc_iron_workload(gb), gb["setup"]["steps"])
    st = o.get_state()
    nm = ckg["nm"]
    template = io.Checkpoint(bytes.fromhex(ckg["simparam_hex"]), [], [], np.zeros(0), np.zeros(0), np.zeros(0),
                             np.array(ckg["ispec"]), bytes.fromhex(ckg["thmsums_hex"]))
    ck = io.checkpoint_from_state(st, template, np.full(nm, 26), np.full(nm, 55.847), np.ones(nm, dtype=int))
    path = tmp_path / "chkp.dat"
    io.write_checkpoint(path, ck)
    back = io.read_checkpoint(path)
    assert len(open(path, "rb").read()) == sum(n + 8 for n in ckg["record_lengths"])
    assert back.simparam == ck.simparam and back.thmsums == ck.thmsums
    for a, b in zip(back.x + back.b, ck.x + ck.b):
        assert np.array_equal(a, b)
    assert np.array_equal(back.ispec, ckg["ispec"]) and np.all(back.atomic_index == 1)
    idx, x, _ = golden_checkpoint_sample(g)
    assert np.max(np.abs(back.x[0][idx] - x[0])) <= 1e-16


def test_checkpoint_rejects_damaged_files(tmp_path):
    p = tmp_path / "bad.dat"
    p.write_bytes(b"\x08\x00\x00\x00" + b"\x00" * 8 + b"\x09\x00\x00\x00")
    with pytest.raises(ValueError):
        io.read_checkpoint(p)
    p.write_bytes(b"\x04\x00\x00\x00abcd\x04\x00\x00\x00")
    with pytest.raises(ValueError):
        io.read_checkpoint(p)


def test_rescale_timestep():
    rng = np.random.default_rng(0)
    x = [rng.normal(size=(5, 3)) for _ in range(4)]
    b = [rng.normal(size=(3, 3)) for _ in range(4)]
    ck = io.Checkpoint(b"", x, b, np.full(5, 26), np.full(5, 55.8), np.ones(5), np.array([26]), b"")
    r = io.rescale_timestep(ck, 1.0, 0.5)
    assert np.array_equal(r.x[0], x[0]) and np.allclose(r.x[1], 0.5 * x[1])
    assert np.allclose(r.x[2], 0.25 * x[2]) and np.allclose(r.b[3], 0.25 * b[3])


def test_system_out_header_is_the_reference_layout():
    """The atom count, the replication line and the box lines of the
    reference's bcc-iron system.out, character for character, from the box
    of its checkpoint; and the 3g14.6 position columns of the sampled atom
    lines from the checkpoint positions."""
    g = io_golden()
    idx, x, b = golden_checkpoint_sample(g)
    nm = g["checkpoint"]["nm"]
    head = io.format_system_out(b[0], np.zeros((0, 3)), [], [], []).split("\n")
    assert io.list_directed_int(nm) == g["system_out_head"][0]
    assert head[1:5] == g["system_out_head"][1:5]
    for k, i in enumerate(idx):
        line = io.format_system_out(b[0], x[0][k:k + 1], [26], [55.847], [-4.0]).split("\n")[5]
        assert line[:42] == g["system_out_positions"][str(i)], i


def test_system_out_round_trip(tmp_path):
    """write_system_out then read_system_out: FORMAT(3g14.6,1X,I3,g12.4,f13.9)
    keeps six significant digits of x0, four of the mass and nine decimals of
    the energy."""
    w = wl.make_workload(3, sigma=0.1, temperature=0.0, seed=4)
    en = np.linspace(-4.3, -3.9, w.nm)
    io.write_system_out(tmp_path / "system.out", w.b0, w.x0, w.atomic_number, w.atomic_mass, en)
    r = io.read_system_out(tmp_path / "system.out")
    assert r["nm"] == w.nm and np.allclose(r["b0"], w.b0, rtol=1e-16, atol=0)
    assert np.allclose(r["x0"], w.x0, rtol=6e-6, atol=1e-12)
    assert np.all(r["atomic_number"] == 26) and np.all(r["atomic_mass"] == float(f"{55.845:.2f}"))
    assert np.allclose(r["en_atom"], en, atol=5e-10)
    lines = open(tmp_path / "system.out").read().splitlines()
    assert all(len(l) == 14 * 3 + 1 + 3 + 12 + 13 for l in lines[5:])


def test_read_system_in_bcc_iron():
    """The reference's 25^3.in: 31,250 atoms, box 25 x 2.87 A, one species,
    positions drawn exactly as the golden run was reproduced."""
    g = io_golden()
    s = io.read_system_in(g["system_in"]["bcc_iron"])
    assert s.nm == 31250 and s.nbasis == 2 and s.nt == (25, 25, 25)
    assert np.allclose(s.b0, np.diag([71.75] * 3), rtol=0, atol=1e-13)
    assert s.ispec == [26] and np.all(s.atomic_index == 1) and np.all(s.atomic_mass == 55.847)
    w = bcc_iron_workload(bcc_iron_golden())
    assert np.array_equal(s.x0, w.x0)


def test_read_system_in_thermal_and_species():
    """The thermal run's system.in (offset basis, unequal box edges), and the
    species numbering of read_system with and without the FETRANSMETAL
    table."""
    g = io_golden()
    s = io.read_system_in(g["system_in"]["thermal"])
    assert s.nm == 2000 and np.allclose(np.diag(s.b0), [28.6, 28.67, 28.75])
    assert np.allclose(s.x0[0], [0.003, 0.002, 0.003]) and np.allclose(s.x0[1], [0.047, 0.0495, 0.051])
    assert np.allclose(s.x0[2], [0.003, 0.002, 0.103])
    text = "3\n1 1 1\n3.0 0 0\n0 3.0 0\n0 0 3.0\n0 0 0 26 55.8\n0.5 0.5 0.5 28 58.7\n0.5 0 0 26 55.8\n"
    s = io.read_system_in(text)
    assert s.ispec == [26, 28] and list(s.atomic_index) == [1, 2, 1]
    s = io.read_system_in(text, fetransmetal=True)
    assert list(s.atomic_index) == [5, 7, 5] and s.nspec == 24
    with pytest.raises(ValueError):
        io.read_system_in(text.replace("28 58.7", "13 27.0"), fetransmetal=True)
    with pytest.raises(ValueError):
        io.read_system_in(text, nspec=3)
    d = io.read_system_in(text, dsp=0.1)
    assert 0 < np.max(np.abs(d.x0 - s.x0)) <= 0.05 / 3.0 + 1e-15
