"""The on-disk formats either side of the hot path, read and written on the
host:

* system.in -- read_system (src/io_m.F90:73-256): basis, replications, box,
  species discovery and the jittered lattice positions;
* system.out -- write_system_out_file (src/io_m.F90:363-379): gfortran
  list-directed header lines and FORMAT(3g14.6,1X,I3,g12.4,f13.9) atom lines;
* the unformatted checkpoint -- read/write_checkpoint_file
  (src/moldin.F90:983-1070): gfortran sequential records with 4-byte length
  markers.  Its first record (simparameters) and last (the thermodynamic
  sums) are derived types in the compiler's layout; they are carried as
  opaque bytes, so a file read here and written back is one the reference
  reads.

A checkpoint or a system file becomes a device state through
:meth:`moldy_b200.system.MoldySystem.set_state` (see :func:`state_arrays`).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

from .workloads import ReferenceRandom

# the species the FETRANSMETAL build fixes (src/io_m.F90:133-136)
FETRANSMETAL_SPECIES = (22, 23, 24, 25, 26, 27, 28, 29, 40, 41, 42, 43, 44, 45, 46, 47,
                        72, 73, 74, 75, 76, 77, 78, 79)


# ------------------------------------------------------------ list-directed
class _Records:
    """List-directed READ over the lines of a file: each READ starts on a
    new line, takes the values it needs (continuing on the following lines
    if one runs short) and leaves the rest of its last line unread."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.pos = 0

    def read(self, n: int, conv):
        out = []
        while len(out) < n:
            if self.pos >= len(self.lines):
                raise ValueError("end of file in list-directed read")
            toks = self.lines[self.pos].replace(",", " ").split()
            self.pos += 1
            for t in toks:
                if len(out) == n:
                    break
                out.append(conv(t))
        return out


def _real(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "e"))


def _int(tok: str) -> int:
    return int(tok)


def list_directed_int(v: int) -> str:
    """gfortran's list-directed default INTEGER: 12 characters."""
    return f"{int(v):12d}"


def _digits(v: float, sig: int):
    """Sign, the sig significant digits and the decimal exponent N with
    |v| = 0.d1d2... x 10**N, rounded to sig digits from the exact value."""
    if v == 0.0:
        return ("-" if np.signbit(v) else ""), "0" * sig, 0
    s = f"{abs(v):.{sig - 1}e}"     # correctly rounded from the exact binary value
    mant, ex = s.split("e")
    return ("-" if v < 0 else ""), mant.replace(".", ""), int(ex) + 1


def list_directed_real8(v: float) -> str:
    """gfortran's list-directed REAL(8) item, G26.17 with E3 exponents: F form
    with 17 significant digits in 21 columns and five trailing blanks for
    0.1 <= |v| < 1e17 (zero too, with 16 decimals), otherwise a 1P E form
    (one digit before the point, 17 after) in 26 columns."""
    sign, dig, n = _digits(v, 17)
    if v == 0.0:
        return f"{sign + '0.' + '0' * 16:>21}" + " " * 5
    if 0 <= n <= 17:
        body = f"{abs(v):.{17 - n}f}"
        return f"{sign + body:>21}" + " " * 5
    sign, dig, n = _digits(v, 18)
    e = n - 1
    return f"{sign}{dig[0]}.{dig[1:]}E{'-' if e < 0 else '+'}{abs(e):03d}".rjust(26)


def g_edit(v: float, w: int, d: int) -> str:
    """Fortran Gw.d output (default exponent): F form in w-4 columns and four
    blanks when 0.1 <= |v| < 10**d after rounding to d digits (and for
    zero), else 0.dddE+ee in w columns."""
    sign, dig, n = _digits(v, d)
    if v == 0.0:
        return f"{0.0:{w - 4}.{d - 1}f}" + " " * 4
    if 0 <= n <= d:
        body = f"{v:.{d - n}f}" + ("." if d == n else "")
        return body.rjust(w - 4) + " " * 4
    ex = f"E{'-' if n < 0 else '+'}{abs(n):02d}" if abs(n) < 100 else f"{'-' if n < 0 else '+'}{abs(n):03d}"
    return f"{sign}0.{dig}{ex}".rjust(w)


# ---------------------------------------------------------------- system.in
@dataclass
class SystemFile:
    """A system.in as read_system builds the state from it."""
    nbasis: int
    nt: tuple
    b0: np.ndarray                 # 3x3, columns are box vectors, scaled by nt
    basis: np.ndarray              # (nbasis, 3) fractional in the unit volume
    atomic_number: np.ndarray      # per atom
    atomic_mass: np.ndarray
    atomic_index: np.ndarray       # 1-based species index per atom
    ispec: list = field(default_factory=list)   # atomic number of each species
    x0: np.ndarray | None = None   # (nm, 3) fractional

    @property
    def nm(self) -> int:
        return len(self.atomic_number)

    @property
    def nspec(self) -> int:
        return len(self.ispec)


def read_system_in(path_or_text, *, dsp: float = 0.0, rng: ReferenceRandom | None = None, nspec: int = 0,
                   fetransmetal: bool = False) -> SystemFile:
    """read_system (src/io_m.F90:73-256).  The basis lines are x y z Z mass;
    species are numbered in order of first appearance (FETRANSMETAL: by the
    fixed 24-element table, every Z must be in it); nspec > 0 must equal the
    count found.  Positions x0 = (rand1() - 1/2) dsp / B0(d,d) + (i0 + xb) /
    nt per direction, three rand1 draws per atom whatever dsp is, in
    x-outer, z-inner, basis-innermost order; rng defaults to the reference's
    rstart(97, 33, 21, 82) generator."""
    text = path_or_text if "\n" in str(path_or_text) else open(path_or_text).read()
    rd = _Records(text)
    (nbasis,) = rd.read(1, _int)
    nt = tuple(rd.read(3, _int))
    b0 = np.zeros((3, 3))
    for i in range(3):
        b0[:, i] = rd.read(3, _real)
    for i in range(3):
        b0[:, i] = b0[:, i] * nt[i]
    basis = np.zeros((nbasis, 3))
    zb = np.zeros(nbasis, dtype=np.int64)
    mb = np.zeros(nbasis)
    for ib in range(nbasis):
        vals = rd.read(5, str)
        basis[ib] = [_real(v) for v in vals[:3]]
        zb[ib] = int(vals[3])
        mb[ib] = _real(vals[4])
    ib_index = np.zeros(nbasis, dtype=np.int64)
    if fetransmetal:
        ispec = list(FETRANSMETAL_SPECIES)
        for z in zb:
            if int(z) not in ispec:
                raise ValueError(f"atomic number {int(z)} is not in the FETRANSMETAL species table")
        ib_index[0] = ispec.index(int(zb[0])) + 1
    else:
        ispec = [int(zb[0])]
        ib_index[0] = 1
    for ib in range(1, nbasis):
        if zb[ib] != zb[ib - 1]:
            if int(zb[ib]) in ispec:
                ib_index[ib] = ispec.index(int(zb[ib])) + 1
            else:
                ispec.append(int(zb[ib]))
                ib_index[ib] = len(ispec)
        else:
            ib_index[ib] = ib_index[ib - 1]
    if nspec > 0 and len(ispec) != nspec:
        raise ValueError("READ_SYSTEM: The number of species found is not equal to NSPEC")
    rng = rng or ReferenceRandom()
    rt = [1.0 / k for k in nt]
    nm = nbasis * nt[0] * nt[1] * nt[2]
    x0 = np.zeros((nm, 3))
    z = np.zeros(nm, dtype=np.int64)
    m = np.zeros(nm)
    idx = np.zeros(nm, dtype=np.int64)
    l = 0
    for i0 in range(nt[0]):
        for j0 in range(nt[1]):
            for k0 in range(nt[2]):
                for ib in range(nbasis):
                    x0[l, 0] = (rng.rand1() - 0.5) * dsp / b0[0, 0] + rt[0] * (i0 + basis[ib, 0])
                    x0[l, 1] = (rng.rand1() - 0.5) * dsp / b0[1, 1] + rt[1] * (j0 + basis[ib, 1])
                    x0[l, 2] = (rng.rand1() - 0.5) * dsp / b0[2, 2] + rt[2] * (k0 + basis[ib, 2])
                    z[l], m[l], idx[l] = zb[ib], mb[ib], ib_index[ib]
                    l += 1
    return SystemFile(nbasis, nt, b0, basis, z, m, idx, ispec, x0)


# --------------------------------------------------------------- system.out
def format_system_out(b0, x0, atomic_number, atomic_mass, en_atom) -> str:
    """write_system_out_file (src/io_m.F90:363-379): the atom count and the
    line "1 1 1" list-directed, the box column by column list-directed, then
    one FORMAT(3g14.6,1X,I3,g12.4,f13.9) line per atom."""
    x0 = np.asarray(x0, dtype=np.float64)
    b0 = np.asarray(b0, dtype=np.float64)
    out = [list_directed_int(len(x0)), " 1 1 1"]
    for i in range(3):
        out.append("".join(list_directed_real8(float(b0[j, i])) for j in range(3)))
    for i in range(len(x0)):
        out.append("".join(g_edit(float(x0[i, d]), 14, 6) for d in range(3)) + " " + f"{int(atomic_number[i]):3d}"
                   + g_edit(float(atomic_mass[i]), 12, 4) + f"{float(en_atom[i]):13.9f}")
    return "\n".join(out) + "\n"


def write_system_out(path, b0, x0, atomic_number, atomic_mass, en_atom):
    with open(path, "w") as f:
        f.write(format_system_out(b0, x0, atomic_number, atomic_mass, en_atom))


def read_system_out(path_or_text) -> dict:
    """A system.out (or any file of its layout): nm, the box, and per atom
    the fractional position, atomic number, mass and energy."""
    text = path_or_text if "\n" in str(path_or_text) else open(path_or_text).read()
    rd = _Records(text)
    (nm,) = rd.read(1, _int)
    rd.read(3, _int)
    b0 = np.zeros((3, 3))
    for i in range(3):
        b0[:, i] = rd.read(3, _real)
    x0 = np.zeros((nm, 3))
    z = np.zeros(nm, dtype=np.int64)
    m = np.zeros(nm)
    en = np.zeros(nm)
    for i in range(nm):
        v = rd.read(6, str)
        x0[i] = [_real(t) for t in v[:3]]
        z[i] = int(v[3])
        m[i] = _real(v[4])
        en[i] = _real(v[5])
    return {"nm": nm, "b0": b0, "x0": x0, "atomic_number": z, "atomic_mass": m, "en_atom": en}


# --------------------------------------------------------------- checkpoint
@dataclass
class Checkpoint:
    """The records of read/write_checkpoint_file (src/moldin.F90:983-1070)."""
    simparam: bytes                # simparameters, compiler layout
    x: list                        # x0, x1, x2, x3: (nm, 3) each
    b: list                        # b0, b1, b2, b3: 3x3 each (columns are box vectors)
    atomic_number: np.ndarray
    atomic_mass: np.ndarray
    atomic_index: np.ndarray
    ispec: np.ndarray
    thmsums: bytes                 # thermodynamic sums, compiler layout

    @property
    def nm(self) -> int:
        return len(self.atomic_number)


def _read_records(data: bytes) -> list:
    out, off = [], 0
    while off < len(data):
        if off + 4 > len(data):
            raise ValueError("truncated record marker")
        (n,) = struct.unpack_from("<i", data, off)
        if n < 0:
            raise ValueError("records of 2 GiB and more (split records) are not supported")
        if off + 8 + n > len(data):
            raise ValueError("truncated record")
        (m,) = struct.unpack_from("<i", data, off + 4 + n)
        if m != n:
            raise ValueError("record markers disagree")
        out.append(data[off + 4:off + 4 + n])
        off += 8 + n
    return out


def _record(payload: bytes) -> bytes:
    if len(payload) >= 2 ** 31 - 9:
        raise ValueError("records of 2 GiB and more (split records) are not supported")
    head = struct.pack("<i", len(payload))
    return head + payload + head


def read_checkpoint(path) -> Checkpoint:
    rec = _read_records(open(path, "rb").read())
    if len(rec) != 10:
        raise ValueError(f"a checkpoint has 10 records, this file {len(rec)}")
    n3 = len(rec[1]) // 8 - 9
    if n3 < 0 or n3 % 3 or any(len(r) != len(rec[1]) for r in rec[2:5]):
        raise ValueError("state records of unequal or invalid length")
    nm = n3 // 3
    x, b = [], []
    for r in rec[1:5]:
        v = np.frombuffer(r, dtype="<f8")
        x.append(np.stack([v[:nm], v[nm:2 * nm], v[2 * nm:3 * nm]], axis=1).copy())
        b.append(v[3 * nm:].reshape(3, 3, order="F").copy())
    zn = np.frombuffer(rec[5], dtype="<i4").astype(np.int64)
    mass = np.frombuffer(rec[6], dtype="<f8").copy()
    aidx = np.frombuffer(rec[7], dtype="<i4").astype(np.int64)
    if len(zn) != nm or len(mass) != nm or len(aidx) != nm:
        raise ValueError("species records do not match the atom count")
    ispec = np.frombuffer(rec[8], dtype="<i4").astype(np.int64)
    return Checkpoint(rec[0], x, b, zn, mass, aidx, ispec, rec[9])


def checkpoint_bytes(ck: Checkpoint) -> bytes:
    nm = ck.nm
    parts = [_record(bytes(ck.simparam))]
    for x, b in zip(ck.x, ck.b):
        x = np.asarray(x, dtype=np.float64).reshape(nm, 3)
        v = np.concatenate([x[:, 0], x[:, 1], x[:, 2], np.asarray(b, dtype=np.float64).ravel(order="F")])
        parts.append(_record(v.astype("<f8").tobytes()))
    parts.append(_record(np.asarray(ck.atomic_number).astype("<i4").tobytes()))
    parts.append(_record(np.asarray(ck.atomic_mass, dtype=np.float64).astype("<f8").tobytes()))
    parts.append(_record(np.asarray(ck.atomic_index).astype("<i4").tobytes()))
    parts.append(_record(np.asarray(ck.ispec).astype("<i4").tobytes()))
    parts.append(_record(bytes(ck.thmsums)))
    return b"".join(parts)


def write_checkpoint(path, ck: Checkpoint):
    with open(path, "wb") as f:
        f.write(checkpoint_bytes(ck))


def rescale_timestep(ck: Checkpoint, old_dt: float, new_dt: float) -> Checkpoint:
    """A restart with a changed timestep (src/moldin.F90:1029-1044): x1, b1
    scale with new/old, x2, b2, x3, b3 with its square."""
    r = new_dt / old_dt
    x = [ck.x[0], ck.x[1] * r, ck.x[2] * r ** 2, ck.x[3] * r ** 2]
    b = [ck.b[0], ck.b[1] * r, ck.b[2] * r ** 2, ck.b[3] * r ** 2]
    return Checkpoint(ck.simparam, x, b, ck.atomic_number, ck.atomic_mass, ck.atomic_index, ck.ispec, ck.thmsums)


def checkpoint_from_state(state: dict, template: Checkpoint, atomic_number, atomic_mass, atomic_index,
                          x3=None, b3=None) -> Checkpoint:
    """A checkpoint of a device state (MoldySystem.get_state(): x0, x1, x2,
    b0, b1, b2), with the compiler-layout records, ispec and the jolt terms
    x3/b3 (zero by default) taken from template."""
    nm = len(state["x0"])
    x3 = np.zeros((nm, 3)) if x3 is None else x3
    b3 = np.zeros((3, 3)) if b3 is None else b3
    return Checkpoint(template.simparam, [state["x0"], state["x1"], state["x2"], x3],
                      [state["b0"], state["b1"], state["b2"], b3], np.asarray(atomic_number),
                      np.asarray(atomic_mass, dtype=np.float64), np.asarray(atomic_index), template.ispec,
                      template.thmsums)


def state_arrays(ck: Checkpoint) -> dict:
    """Keyword arguments for MoldySystem.set_state from a checkpoint."""
    return {"x0": ck.x[0], "x1": ck.x[1], "x2": ck.x[2], "b0": ck.b[0], "b1": ck.b[1], "b2": ck.b[2],
            "atomic_number": ck.atomic_number, "atomic_mass": ck.atomic_mass}
