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
