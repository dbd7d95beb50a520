"""Shared helpers for the parity tests: run the oracle and the GPU library on
the same seeded inputs and compare with written tolerances."""
from __future__ import annotations

import numpy as np


def real_forces(f_frac: np.ndarray, b0: np.ndarray) -> np.ndarray:
    """Real forces B0 f in eV/A (src/dynamics_m.F90:603-606)."""
    return f_frac @ np.asarray(b0).T


def rel_norm_err(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / max(||b||, tiny): a norm-wise relative error."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / max(nb, 1e-300))


def pair_set(nlist: np.ndarray, numn: np.ndarray) -> set:
    """Unordered pair set of a half list (1-based entries)."""
    s = set()
    for i in range(len(numn)):
        for j in nlist[i, :numn[i]]:
            a, b = i + 1, int(j)
            s.add((a, b) if a < b else (b, a))
    return s


def perturb(w, rng, amp_frac: float):
    """Random fractional displacements (uniform, +/- amp_frac) of a workload copy."""
    w2 = w.copy()
    w2.x0 = w2.x0 + rng.uniform(-amp_frac, amp_frac, size=w2.x0.shape)
    return w2


def bcc_iron_golden():
    import json
    import os
    return json.load(open(os.path.join(os.path.dirname(__file__), "golden", "bcc_iron_step10.json")))


def bcc_iron_workload(g):
    """The reference's shipped bcc-iron run: read_system's 25^3 bcc lattice
    (a0 = 2.87 A) drawing its three rand1 numbers per atom, then setvel at
    600 K from the same generator (rstart(97,33,21,82)); PR NPT at 0.1 GPa,
    box mass 50, dt 1 fs, rnear = 5.4 + 1.0 A, 3^3 link cells."""
    from moldy_b200 import workloads as wl
    s = g["setup"]
    n = s["cells"]
    w = wl.make_workload(n, a0=s["a0"], sigma=0.0, temperature=0.0, ivol=0, press_gpa=s["press_GPa"],
                         boxmass=s["boxmass"], dt_fs=s["dt_fs"], rpad=s["rpad"], nbrupdate=s["nbrupdate"],
                         nnbrs=s["nnbrs"], seed=1, name="bcc_iron_reference_run")
    w.rnear = 5.4 + s["rpad"]
    w.nlc = tuple(s["nlc"])
    w.atomic_mass = np.full(w.nm, s["mass"])
    w.del2 = w.deltat ** 2 / (2.0 * w.atomic_mass)
    rng = wl.ReferenceRandom(*s["rstart"])
    w.x0 = wl.read_system_positions(n, rng, dsp=0.0, b0=w.b0)
    return wl.setvel_reference(w, s["temprq_K"], rng)


def printed_tolerance(text: str) -> float:
    """Half a unit in the last printed digit of a number as printed."""
    t = text.strip().upper()
    mant, _, exp = t.partition("E")
    dec = len(mant.split(".")[1]) if "." in mant else 0
    return 0.5 * 10.0 ** (-dec + (int(exp) if exp else 0))


def check_against_bcc_iron_golden(g, thermo, stress_no_ke, b0, x0, en_atom):
    """Asserts agreement with every printed digit of the golden run."""
    for k, text in g["thermo_step10"].items():
        v = {"PE": thermo["pe"], "KE": thermo["ke"], "TE": thermo["te"], "T": thermo["temp"],
             "H": thermo["h"], "TH": thermo["th"], "VOL": thermo["vol"]}[k]
        assert abs(v - float(text)) <= printed_tolerance(text) * 1.0001, (k, v, text)
    for i in range(3):
        for j in range(3):
            text = g["stress_no_ke_GPa"][i][j]
            assert abs(stress_no_ke[i, j] - float(text)) <= printed_tolerance(text) * 1.0001, (i, j)
    bref = np.array([[float(v) for v in col] for col in g["box_columns"]]).T
    assert np.max(np.abs(b0 - bref)) <= 1e-12 * 71.75
    for k, idx in enumerate(g["sample_index"]):
        for c in range(3):
            text = g["sample_x0"][k][c]
            assert abs(x0[idx, c] - float(text)) <= printed_tolerance(text) * 1.0001, (idx, c)
        if en_atom is not None:
            text = g["sample_en_atom"][k]
            assert abs(en_atom[idx] - float(text)) <= printed_tolerance(text) * 1.0001, (idx, "en")
