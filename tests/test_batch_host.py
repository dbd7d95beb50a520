"""Host logic of the sharded batch: per-system results gathered from two
gloo ranks (torch.distributed on CPU) land at their global indices on every
rank."""
import os
import socket

import numpy as np

from moldy_b200.adjoint import shard_configs
from moldy_b200.batch import gather_system_results


def _fake_results(idx):
    idx = np.asarray(idx, dtype=np.float64)
    return {"pe": -4.0 * idx, "tp": np.stack([np.eye(3) * (i + 0.5) for i in idx]) if len(idx) else np.zeros((0, 3, 3)),
            "iflag": (idx % 3).astype(np.float64)}


def _rank_main(rank, world, port, natoms, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assignment = shard_configs(natoms, world)
        got = gather_system_results(_fake_results(assignment[rank]), assignment, len(natoms))
        np.savez(out % rank, **got)
    finally:
        dist.destroy_process_group()


def test_gather_system_results_gloo(tmp_path):
    import torch.multiprocessing as mp
    natoms = [128, 8192, 1024, 2000, 250, 686, 3456, 54, 432]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "r%d.npz")
    mp.start_processes(_rank_main, args=(2, port, natoms, out), nprocs=2, join=True, start_method="spawn")
    want = _fake_results(range(len(natoms)))
    for r in range(2):
        got = np.load(out % r)
        for k, v in want.items():
            assert np.array_equal(got[k], v), (r, k)


def test_gather_without_process_group():
    got = gather_system_results(_fake_results([0, 1, 2]), [[0, 1, 2]], 3)
    assert np.array_equal(got["pe"], [0.0, -4.0, -8.0])
