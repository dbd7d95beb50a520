"""Writes tests/golden/bcc_iron_rdf.json from the radial distribution
function the reference ships with its bcc-iron run
(tests/reference/bcc_iron/rdf.dat in the reference project): the pair count
of each of the 500 bins of 0.02 A, written by rdf(500, 50) at the end of the
10-step run.  That file comes from the routine's older form, which binned
every pair of atoms; its lines read "BIN, NO IN BINS <bin> <count>".

Run once where the reference is available:
    python tests/golden/make_bcc_iron_rdf_golden.py /path/to/reference
"""
import json
import os
import sys


def main(ref_root):
    path = os.path.join(ref_root, "tests", "reference", "bcc_iron", "rdf.dat")
    counts = []
    for line in open(path):
        f = line.split()
        if not f:
            continue
        assert int(f[-2]) == len(counts) + 1, line
        counts.append(int(f[-1]))
    golden = {
        "source": "tests/reference/bcc_iron/rdf.dat of the reference (rdf(500, 50), older all-pairs form)",
        "maxbin": 500, "binsperangstrom": 50,
        "counts": counts,
    }
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bcc_iron_rdf.json")
    json.dump(golden, open(out, "w"), separators=(",", ":"))
    print(out, len(counts), sum(counts))


if __name__ == "__main__":
    main(sys.argv[1])
