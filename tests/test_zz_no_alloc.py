"""moldy_gpu_force_noalloc: the force evaluation for callers that cannot
allocate device memory (their buffers come from another allocator, or the
code must not allocate while it runs).

The test owns every device buffer (torch tensors), calls the entry point
through the C ABI twice in a row, and checks both results against the
existing moldy_gpu_force on the same configuration.  The file name makes
pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

from moldy_b200 import workloads as wl
from tests.helpers import rel_norm_err

pytestmark = pytest.mark.gpu

TOL = 1e-10   # same FP64 parity bound as the other force tests


def _setup(gpu_lib):
    """A 2000-atom configuration whose tables the caller supplies (the
    FETRANSMETAL Fe-Fe functions over [rmin, rmax] = [0.5, 6.0] A): the same
    tables and ranges go to both entry points."""
    import oracle
    from moldy_b200 import MoldySystem
    w = wl.make_workload(10, sigma=0.08, temperature=0.0, seed=17)   # 2000 atoms
    o = oracle.from_workload(w, uselookup=True, threads=1)
    rng = dict(rmin=0.5, rmax=6.0, rhomin=0.0, rhomax=10000.0)
    n = 5000
    r = rng["rmin"] + np.arange(n + 1) * ((rng["rmax"] - rng["rmin"]) / n)
    tab = {k: np.array([o.src(i, x) for x in r]) for i, k in enumerate(("vee", "dvee", "phi", "dphi"))}
    full = o.tables()
    tab["emb"], tab["demb"] = full["emb"], full["demb"]
    o.close()
    g = MoldySystem(w.nm, rnear=w.rnear, deltat=w.deltat, ivol=w.ivol, ntcm=w.ntcm, nlc=w.nlc)
    g.set_tables(tab, **rng)
    g.set_state(w.x0, w.x1, w.x2, w.b0, w.b1, w.b2, w.atomic_number, w.atomic_mass, w.del2)
    return w, g, tab, rng


def _device_args(w, nlist, numn, tab):
    import torch
    dev = torch.device("cuda", 0)
    t64 = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    d = {
        "x": [t64(w.x0[:, k]) for k in range(3)],
        "mass": t64(w.atomic_mass),
        "nlist": torch.as_tensor(np.ascontiguousarray(nlist), dtype=torch.int32, device=dev),
        "numn": torch.as_tensor(np.ascontiguousarray(numn), dtype=torch.int32, device=dev),
        "tabs": [t64(tab[k]) for k in ("vee", "dvee", "phi", "dphi", "emb", "demb")],
        "f": [torch.empty(w.nm, dtype=torch.float64, device=dev) for _ in range(3)],
        "ev": torch.empty(10, dtype=torch.float64, device=dev),
        "stream": torch.cuda.current_stream(dev),
    }
    return d


def _call(L, w, d, tab, rng):
    from moldy_b200 import _lib
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    b0 = np.ascontiguousarray(w.b0.ravel(order="F"))
    return L.moldy_gpu_force_noalloc(
        w.nm, w.nnbrs, w.ivol, ptr(d["x"][0]), ptr(d["x"][1]), ptr(d["x"][2]), ptr(d["mass"]),
        b0.ctypes.data_as(_lib.D), ptr(d["nlist"]), ptr(d["numn"]), len(tab["vee"]) - 1,
        rng["rmin"], rng["rmax"], rng["rhomin"], rng["rhomax"], *[ptr(t) for t in d["tabs"]],
        *[ptr(t) for t in d["f"]], ptr(d["ev"]), ctypes.c_void_p(d["stream"].cuda_stream))


def test_force_noalloc_matches_force(gpu_lib):
    import torch
    from moldy_b200 import _lib

    L = _lib.load()
    w, g, tab, rng = _setup(gpu_lib)
    ref = g.force()
    f_ref = g.forces()
    nlist, numn = g.neighbour_list()          # NLIST(nnbrs, nm), 1-based
    d = _device_args(w, nlist, numn, tab)
    for _ in range(2):
        rc = _call(L, w, d, tab, rng)
        assert rc == 0, L.moldy_gpu_last_error()
        torch.cuda.synchronize()
        f_got = np.stack([t.cpu().numpy() for t in d["f"]], axis=1)
        out = d["ev"].cpu().numpy()
        assert rel_norm_err(f_got, f_ref) < TOL
        assert abs(out[0] - ref["pe"]) < TOL * abs(ref["pe"])
        assert rel_norm_err(out[1:].reshape(3, 3, order="F"), ref["tp"]) < TOL


def test_force_noalloc_reports_malformed_lists(gpu_lib):
    """An NLIST entry outside 1..nm, or a NUMN count outside 0..nnbrs, is
    skipped or clamped on the device (every access stays in bounds) and the
    call returns MOLDY_ERR_INVALID with its own message."""
    import torch
    from moldy_b200 import _lib

    L = _lib.load()
    w, g, tab, rng = _setup(gpu_lib)
    g.force()
    nlist, numn = g.neighbour_list()
    bad = nlist.copy()
    bad[5, 0] = w.nm + 1
    d = _device_args(w, bad, numn, tab)
    assert _call(L, w, d, tab, rng) == 1                      # MOLDY_ERR_INVALID
    assert b"outside 1..nm" in L.moldy_gpu_last_error()
    torch.cuda.synchronize()
    assert all(bool(torch.isfinite(t).all()) for t in d["f"])
    badn = numn.copy()
    badn[7] = w.nnbrs + 3
    d = _device_args(w, nlist, badn, tab)
    assert _call(L, w, d, tab, rng) == 1
    assert b"NUMN" in L.moldy_gpu_last_error()
    torch.cuda.synchronize()
    assert all(bool(torch.isfinite(t).all()) for t in d["f"])


def test_force_noalloc_rejects_oversize(gpu_lib):
    from moldy_b200 import _lib
    L = _lib.load()
    z = ctypes.c_void_p(0)
    b0 = np.eye(3).ravel()
    rc = L.moldy_gpu_force_noalloc(_lib.NOALLOC_MAX_ATOMS + 1, 150, 1, z, z, z, z,
                                   b0.ctypes.data_as(_lib.D), z, z, 5000, 0.0, 6.0, 0.0, 1e4,
                                   *([z] * 6), z, z, z, z, z)
    assert rc == 6
    assert b"MOLDY_NOALLOC_MAX_ATOMS" in L.moldy_gpu_last_error()
