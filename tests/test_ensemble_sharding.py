"""Ensemble sharding over ranks (CPU, gloo): every domain lands on exactly one rank, loads balance, and
rank 0 receives every domain's result once."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_partition_covers_every_domain_once_and_balances():
    from wspm_b200.ensemble import partition_domains
    rng = np.random.default_rng(0)
    work = 7 * (rng.choice(np.arange(32, 257, 16), 256) + 1) ** 2
    for world in (1, 2, 3, 8):
        parts = partition_domains(work, world)
        ids = np.concatenate(parts)
        assert np.array_equal(np.sort(ids), np.arange(256))
        loads = np.array([work[p].sum() for p in parts])
        assert loads.max() - loads.min() <= work.max()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, out_path):
    import torch.distributed as dist
    from wspm_b200.ensemble import gather_domain_results, partition_domains
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        work = np.arange(1, n + 1) ** 2
        mine = partition_domains(work, world)[rank]
        vals = 1000 + mine                      # each rank "solves" its domains
        got = gather_domain_results(mine, vals, n, world)
        if rank == 0:
            np.save(out_path, got)
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


def test_gather_on_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    n, world = 37, 2
    out = str(tmp_path / "gathered.npy")
    mp.spawn(_worker, args=(world, _free_port(), n, out), nprocs=world, join=True)
    np.testing.assert_array_equal(np.load(out), 1000 + np.arange(n))
