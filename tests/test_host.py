"""Host-side tests (no GPU): the C-ABI library loads and exports every entry
point its header declares, the product refuses to run without a GPU, the
synthetic workloads and the coefficient reader."""
import os
import re

import numpy as np
import pytest

from moldy_b200 import potentials, units
from moldy_b200 import workloads as wl

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "moldy_gpu.h")).read()
    return sorted(set(re.findall(r"\b(moldy_(?:gpu|fetm|ic)_[a-z_0-9]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    from moldy_b200 import build, _lib
    build.build()
    lib = _lib.load()
    names = _declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES)
    assert lib.moldy_gpu_version().decode().startswith("moldy_b200")


def test_library_is_built_for_sm100a():
    """The shared object carries sm_100a code (checked from the build recipe)."""
    from moldy_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_no_gpu_fails_loudly():
    from moldy_b200 import MoldySystem, MoldyError
    with pytest.raises(MoldyError) as ei:
        MoldySystem(16)
    assert ei.value.code == 8


def test_invalid_params_rejected_before_device():
    import ctypes
    from moldy_b200 import _lib
    L = _lib.load()
    p = _lib.Params(rnear=6.3, deltat=0.1, nm=0, nnbrs=150, ivol=1, ntcm=10)
    h = _lib.H()
    assert L.moldy_gpu_create(ctypes.byref(p), ctypes.byref(h)) == 1
    assert b"nm" in L.moldy_gpu_last_error()
    p.nm, p.nlcx, p.nlcy, p.nlcz = 10, 2, 3, 3
    assert L.moldy_gpu_create(ctypes.byref(p), ctypes.byref(h)) == 1


def test_bcc_lattice_layout():
    x = wl.bcc_fractional(3)
    assert x.shape == (54, 3)
    # read_system order: x replicas outermost, then y, z, then the basis
    assert np.allclose(x[0], 0) and np.allclose(x[1], [1 / 6] * 3)
    assert np.allclose(x[2], [0, 0, 1 / 3])
    assert np.allclose(x[6], [0, 1 / 3, 0]) and np.allclose(x[18], [1 / 3, 0, 0])


def test_workload_temperature_and_units():
    w = wl.make_workload(6, temperature=600.0, sigma=0.0, seed=3)
    v = (w.x1 @ w.b0.T) / w.deltat
    ke = 0.5 * np.sum(w.atomic_mass[:, None] * v * v)
    assert abs(ke - 1.5 * units.BK * 600.0 * (w.nm - 1)) < 1e-9 * ke
    assert np.allclose((w.atomic_mass[:, None] * v).sum(0), 0.0, atol=1e-9)
    assert abs(w.deltat - 0.098227) < 1e-6                      # 1 fs in model units
    assert abs(units.PRESS_TO_GPA - 160.2176) < 1e-3
    assert w.nlc == (3, 3, 3)


def test_link_cell_counts_match_moldin():
    b0 = np.diag([286.65, 100.0, 18.0])
    assert wl.link_cell_counts(b0, 6.3) == (45, 15, 3)


def test_pot_file_reader():
    c = potentials.read_pot_file(os.path.join(ROOT, "tests", "golden", "pot_026_026.in"))
    f = potentials.FE_FE
    for a, b in ((c.av, f.av), (c.rv, f.rv), (c.ap, f.ap), (c.rp, f.rp)):
        assert np.array_equal(a, b)
    assert c.rmax == 3.72645


def test_strain_is_symmetric():
    rng = np.random.default_rng(0)
    e = wl.random_symmetric_strain(rng, 0.02)
    assert np.allclose(e, e.T) and np.max(np.abs(e)) <= 0.02
