"""Generates the known-answer fixtures in tests/golden/ (run from the repo root).

perfect_lattice.json: energy per atom, density and lattice forces of perfect
bcc Fe for the FETRANSMETAL Fe-Fe coefficients (pot_026_026.in), evaluated
analytically at 30 significant digits with mpmath.  For a perfect bcc
lattice the first shell has 8 neighbours at a0*sqrt(3)/2 and the second 6 at
a0; the third shell (a0*sqrt(2) = 4.05 A) lies beyond every knot, so

    rho = 8 phi(r1) + 6 phi(r2),   E/atom = F(rho) + (8 V(r1) + 6 V(r2)) / 2,

with F(rho) = -sqrt(rho).  These are independent of any lookup table; the
tabulated values differ by the interpolation error, which the tests bound.

pot_026_026.in: the coefficient file in the reference's fixed format, used to
test the reader without touching the reference tree.
"""
from __future__ import annotations

import json
import os
import sys

from mpmath import mp, mpf, sqrt

sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..", "..")))
from moldy_b200.potentials import FE_FE  # noqa: E402

mp.dps = 30
HERE = os.path.dirname(os.path.abspath(__file__))


def cubic_sum(amps, knots, r):
    s = mpf(0)
    for a, k in zip(amps, knots):
        d = mpf(repr(float(k))) - r
        if d >= 0:
            s += mpf(repr(float(a))) * d ** 3
    return s


def dcubic_sum(amps, knots, r):
    s = mpf(0)
    for a, k in zip(amps, knots):
        d = mpf(repr(float(k))) - r
        if d >= 0:
            s -= 3 * mpf(repr(float(a))) * d ** 2
    return s


def perfect(a0: str):
    a = mpf(a0)
    r1, r2 = a * sqrt(3) / 2, a
    c = FE_FE
    rho = 8 * cubic_sum(c.ap, c.rp, r1) + 6 * cubic_sum(c.ap, c.rp, r2)
    e = -sqrt(rho) + (8 * cubic_sum(c.av, c.rv, r1) + 6 * cubic_sum(c.av, c.rv, r2)) / 2
    # pressure-like radial derivative dE/da per atom, for the stress sign check
    dF = -1 / (2 * sqrt(rho))
    drho = 8 * dcubic_sum(c.ap, c.rp, r1) * sqrt(3) / 2 + 6 * dcubic_sum(c.ap, c.rp, r2)
    dV = (8 * dcubic_sum(c.av, c.rv, r1) * sqrt(3) / 2 + 6 * dcubic_sum(c.av, c.rv, r2)) / 2
    return {"a0": float(a), "rho": float(rho), "e_per_atom": float(e),
            "de_da_per_atom": float(dF * drho + dV), "r1": float(r1), "r2": float(r2)}


def main():
    out = {"source": "FETRANSMETAL Fe-Fe knots of pot_026_026.in, mpmath 30 digits",
           "cases": [perfect("2.8665"), perfect("2.870"), perfect("2.80"), perfect("2.95")]}
    with open(os.path.join(HERE, "perfect_lattice.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    c = FE_FE
    lines = ["# AVTF format coefficients for cubic spline material potential #",
             "26        # Principal Atomic number", "26        # Second Atomic number",
             f"{len(c.av)}         # Number of coefficients (vee)",
             f"{len(c.ap)}         # Number of coefficients (phi)",
             f"{c.rmin}       # Minimum potential radius", f"{c.rmax}   # Maximum potential radius",
             " ".join(repr(float(v)) for v in c.av) + " # a_k coefficients (vee)",
             " ".join(repr(float(v)) for v in c.rv) + " # r_k coefficients (vee)",
             " ".join(repr(float(v)) for v in c.ap) + " # a_k coefficients (phi)",
             " ".join(repr(float(v)) for v in c.rp) + " # r_k coefficients (phi)",
             "# END OF INPUT #"]
    with open(os.path.join(HERE, "pot_026_026.in"), "w") as fh:
        fh.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
