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


def test_force_noalloc_matches_force(gpu_lib):
    import torch
    from moldy_b200 import MoldySystem, _lib

    L = _lib.load()
    w = wl.make_workload(10, sigma=0.08, temperature=0.0, seed=17)   # 2000 atoms
    g = MoldySystem.from_workload(w)
    ref = g.force()
    f_ref = g.forces()
    nlist, numn = g.neighbour_list()          # NLIST(nnbrs, nm), 1-based
    tab = g.tables()

    dev = torch.device("cuda", 0)
    t64 = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    x = [t64(w.x0[:, k]) for k in range(3)]
    mass = t64(w.atomic_mass)
    d_nlist = torch.as_tensor(np.ascontiguousarray(nlist), dtype=torch.int32, device=dev)
    d_numn = torch.as_tensor(numn, dtype=torch.int32, device=dev)
    tabs = [t64(tab[k]) for k in ("vee", "dvee", "phi", "dphi", "emb", "demb")]
    f = [torch.empty(w.nm, dtype=torch.float64, device=dev) for _ in range(3)]
    ev = torch.empty(10, dtype=torch.float64, device=dev)
    b0 = np.ascontiguousarray(w.b0.ravel(order="F"))
    stream = torch.cuda.current_stream(dev)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())

    for _ in range(2):
        rc = L.moldy_gpu_force_noalloc(
            w.nm, w.nnbrs, w.ivol, ptr(x[0]), ptr(x[1]), ptr(x[2]), ptr(mass),
            b0.ctypes.data_as(_lib.D), ptr(d_nlist), ptr(d_numn), len(tab["vee"]) - 1,
            0.0, 6.0, 0.0, 10000.0, *[ptr(t) for t in tabs], *[ptr(t) for t in f], ptr(ev),
            ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.moldy_gpu_last_error()
        torch.cuda.synchronize()
        f_got = np.stack([t.cpu().numpy() for t in f], axis=1)
        out = ev.cpu().numpy()
        assert rel_norm_err(f_got, f_ref) < TOL
        assert abs(out[0] - ref["pe"]) < TOL * abs(ref["pe"])
        assert rel_norm_err(out[1:].reshape(3, 3, order="F"), ref["tp"]) < TOL


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
