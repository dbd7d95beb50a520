"""Writes tests/golden/bcc_iron_step10.json from the reference's shipped
bcc-iron run (tests/reference/bcc_iron in the reference project): the
thermodynamics, stress and box printed at step 10 (output66.txt), the final
box and a sample of the final positions and per-atom energies (system.out),
and the tabulated Fe-Fe functions of the IRON_CARBON module (potential.55).

Run once where the reference is available:
    python tests/golden/make_bcc_iron_golden.py /path/to/reference
"""
import json
import os
import re
import sys

SAMPLE_STRIDE = 61


def main(ref_root):
    d = os.path.join(ref_root, "tests", "reference", "bcc_iron")
    out = open(os.path.join(d, "output66.txt")).read()
    out = out[out.index("RUNNING AVERAGES AT STEP NO."):]      # the step-10 block

    def grab(label):
        m = re.search(r"^\s*" + re.escape(label) + r":\s+(\S+)", out, re.M)
        return m.group(1)

    thermo = {k: grab(k) for k in ("PE", "KE", "TE", "T", "H", "TH", "VOL")}
    stress = []
    for i in (1, 2, 3):
        m = re.search(r"STRESS I=\s*%d\s+(\S+)\s+(\S+)\s+(\S+) GPa" % i, out)
        stress.append(list(m.groups()))
    lines = open(os.path.join(d, "system.out")).read().splitlines()
    nm = int(lines[0].split()[0])
    cols = [[v for v in lines[2 + i].split()] for i in range(3)]     # column i of B0 per line
    atoms = [l.split() for l in lines[5:5 + nm]]
    sample = list(range(0, nm, SAMPLE_STRIDE)) + [nm - 1]
    pot = [l.split() for l in open(os.path.join(d, "potential.55")).read().splitlines() if l.strip()]
    golden = {
        "source": "tests/reference/bcc_iron of the reference (output66.txt step 10, system.out, potential.55)",
        "setup": {"cells": 25, "a0": 2.87, "basis": [[0, 0, 0], [0.5, 0.5, 0.5]], "mass": 55.847,
                  "temprq_K": 600.0, "press_GPa": 0.1, "boxmass": 50.0, "dt_fs": 1.0, "rpad": 1.0,
                  "nlc": [3, 3, 3], "nnbrs": 150, "nbrupdate": 2000, "steps": 10,
                  "rstart": [97, 33, 21, 82], "potential": "IRON_CARBON Fe-Fe, lookup nlookup=5000"},
        "thermo_step10": thermo,
        "stress_no_ke_GPa": stress,
        "box_columns": cols,
        "atoms": nm,
        "sample_index": sample,
        "sample_x0": [atoms[i][0:3] for i in sample],
        "sample_en_atom": [atoms[i][5] for i in sample],
        "sum_x0_printed": [repr(sum(float(a[c]) for a in atoms)) for c in range(3)],
        "potential55": pot,
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bcc_iron_step10.json")
    with open(dst, "w") as fh:
        json.dump(golden, fh, indent=0)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
