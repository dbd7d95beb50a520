"""Writes tests/golden/bcc_iron_io.json from the reference's shipped test
runs (tests/reference in the reference project):

* the system.in files of the bcc-iron (25^3.in) and thermal runs, verbatim;
* the first five lines of the bcc-iron system.out (atom count, replication
  line and box, in gfortran list-directed layout) and the position columns
  (3g14.6) of a sample of its atom lines;
* from the bcc-iron unformatted checkpoint chkp_out.dat: every record
  length, the compiler-layout simparameters and thermodynamic-sum records as
  hex, the ispec record, the four box matrices and, for a sample of atoms,
  x0..x3, atomic number, mass and species index at full precision (as
  float.hex strings).

Run once where the reference is available:
    python tests/golden/make_bcc_iron_io_golden.py /path/to/reference
"""
import json
import os
import struct
import sys

STRIDE = 251


def records(path):
    data = open(path, "rb").read()
    out, off = [], 0
    while off < len(data):
        (n,) = struct.unpack_from("<i", data, off)
        out.append(data[off + 4:off + 4 + n])
        off += 8 + n
    return out


def main(ref_root):
    base = os.path.join(ref_root, "tests", "reference")
    bcc = os.path.join(base, "bcc_iron")
    sys_in = {"bcc_iron": open(os.path.join(bcc, "25^3.in")).read(),
              "thermal": open(os.path.join(base, "thermal", "system.in")).read()}
    out_lines = open(os.path.join(bcc, "system.out")).read().split("\n")
    nm = int(out_lines[0].split()[0])
    sample = list(range(0, nm, STRIDE)) + [nm - 1]
    rec = records(os.path.join(bcc, "chkp_out.dat"))
    assert (len(rec[1]) // 8 - 9) % 3 == 0 and (len(rec[1]) // 8 - 9) // 3 == nm
    state = []
    for r in rec[1:5]:
        v = struct.unpack("<%dd" % (len(r) // 8), r)
        state.append(v)
    zn = struct.unpack("<%di" % nm, rec[5])
    mass = struct.unpack("<%dd" % nm, rec[6])
    aidx = struct.unpack("<%di" % nm, rec[7])
    ispec = struct.unpack("<%di" % (len(rec[8]) // 4), rec[8])
    atoms = {}
    for i in sample:
        atoms[str(i)] = {"x": [[float.hex(st[d * nm + i]) for d in range(3)] for st in state],
                         "z": zn[i], "mass": float.hex(mass[i]), "index": aidx[i]}
    golden = {
        "source": "tests/reference/{bcc_iron,thermal} of the reference (system.in, system.out, chkp_out.dat)",
        "system_in": sys_in,
        "system_out_head": out_lines[:5],
        "system_out_positions": {str(i): out_lines[5 + i][:42] for i in sample},
        "checkpoint": {
            "record_lengths": [len(r) for r in rec],
            "nm": nm,
            "simparam_hex": rec[0].hex(),
            "thmsums_hex": rec[9].hex(),
            "ispec": list(ispec),
            "boxes": [[float.hex(v) for v in st[3 * nm:]] for st in state],
            "atoms": atoms,
        },
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bcc_iron_io.json")
    json.dump(golden, open(path, "w"), separators=(",", ":"))
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main(sys.argv[1])
