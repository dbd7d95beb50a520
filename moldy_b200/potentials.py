"""FETRANSMETAL Fe-Fe potential coefficients and the ``pot_XX_YY.in`` reader.

The Hepburn-Ackland-Olsson Fe-Fe potential of the reference's default build
(``src/fetransmetal.F90``) is a sum of cubic knots:

* pair term  V(r)   = sum_k a_k (r_k - r)^3 H(r_k - r)   (6 knots, r > 1.9 A),
* density    phi(r) = sum_k A_k (R_k - r)^3 H(R_k - r)   (2 knots),
* embedding  F(rho) = -sqrt(rho).

The knot values below are the physical parameters of that potential as given
in the reference's data file ``src/potentials/pot_026_026.in`` (lines 7-10);
they must be identical for the energies to be the same.  ``read_pot_file``
parses a file in that fixed format (``src/fetransmetal.F90:603-766``).
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass(frozen=True)
class FeFeCoefficients:
    av: np.ndarray   # pair-term amplitudes a_k (eV/A^3)
    rv: np.ndarray   # pair-term knots r_k (A)
    ap: np.ndarray   # density amplitudes A_k
    rp: np.ndarray   # density knots R_k (A)
    rmin: float = 0.0
    rmax: float = 3.72645


FE_FE = FeFeCoefficients(
    av=np.array([-1.5522046829558238, 2.649967308467956, -0.5585432738234233,
                 -0.11554019572462691, 0.37200356634895027, 4.245653512216868]),
    rv=np.array([3.38247, 3.296475, 3.09582, 2.837835, 2.665845, 2.4824606625]),
    ap=np.array([3.093738340374042, -4.285763262]),
    rp=np.array([3.72645, 3.4398000]),
)


def _numbers(line: str, count: int) -> list[float]:
    toks = line.split("#", 1)[0].split()
    return [float(t.replace("d", "e").replace("D", "e")) for t in toks[:count]]


def read_pot_file(path: str) -> FeFeCoefficients:
    """Reads a ``pot_XX_YY.in`` coefficient file (fixed line order)."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    # line 1 title; 2,3 atomic numbers; 4,5 coefficient counts; 6,7 rmin/rmax;
    # 8-11 a_v, r_v, a_p, r_p
    nv = int(_numbers(lines[3], 1)[0])
    np_ = int(_numbers(lines[4], 1)[0])
    rmin = _numbers(lines[5], 1)[0]
    rmax = _numbers(lines[6], 1)[0]
    av = _numbers(lines[7], nv)
    rv = _numbers(lines[8], nv)
    ap = _numbers(lines[9], np_)
    rp = _numbers(lines[10], np_)
    if len(av) != nv or len(rv) != nv or len(ap) != np_ or len(rp) != np_:
        raise ValueError(f"malformed potential file {path}")
    return FeFeCoefficients(np.array(av), np.array(rv), np.array(ap), np.array(rp), rmin, rmax)
