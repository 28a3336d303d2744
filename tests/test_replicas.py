"""Multi-process path of bench.py on CPU: world-size-2 gloo ranks, each with its
own scenario (seed = rank), combined as independent replicas (no data-path
collective): whole-job throughput = particles of all ranks x steps / the
slowest rank's time."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import gcs
        # each rank builds its own replica scenario from its rank seed
        stars = gcs.collision_equal(*bench.counts_for(45056), seed=rank)
        digest = float(np.float64(stars["x"]).sum())
        n_local = 1000 * (rank + 1)
        value, t_max, n_all = bench.replica_throughput(n_local, 3, 0.5 + rank, dist, "cpu")
        out[rank] = (value, t_max, n_all, len(stars), digest)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_over_two_gloo_ranks(gcs_mod):
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        value, t_max, n_all, n, _ = res[r]
        assert t_max == pytest.approx(1.5)        # the slowest rank's time
        assert n_all == 3000                       # particles of both ranks
        assert value == pytest.approx(3000 * 3 / 1.5)
        assert n == 45056
    assert res[0][4] != res[1][4]                  # different scenarios per rank


def test_replica_throughput_single_process():
    import bench
    value, t, n = bench.replica_throughput(500, 4, 2.0)
    assert (value, t, n) == (1000.0, 2.0, 500)


def _shard_main(rank, world, port, out):
    import datetime
    import torch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        n = 1000
        length, slices = bench.shard_slices(n, world, 64)
        full = torch.full((world * length, 4), -1.0)
        first, count = slices[rank]
        full[first:first + count] = float(rank + 1)
        bench.allgather_slices(dist, full, length, rank)
        out[rank] = (length, slices, full[:n, 0].tolist())
    finally:
        dist.destroy_process_group()


def test_shard_slices_and_allgather_over_two_gloo_ranks():
    """One scenario across ranks: group-aligned equal slices, and after the
    all-gather every rank holds every rank's slice."""
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_shard_main, args=(world, _free_port(), out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    for r in range(world):
        length, slices, rows = res[r]
        assert length == 512 and slices == [(0, 512), (512, 488)]
        assert rows[:512] == [1.0] * 512 and rows[512:] == [2.0] * 488


def test_shard_slices_edge_cases():
    import bench
    assert bench.shard_slices(100, 1, 64) == (128, [(0, 100)])
    length, sl = bench.shard_slices(70, 4, 32)
    assert length == 32 and sl == [(0, 32), (32, 32), (64, 6), (70, 0)]
    assert sum(c for _, c in sl) == 70
