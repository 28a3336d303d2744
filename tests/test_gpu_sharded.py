"""One scenario stepped across devices, emulated on one GPU: two contexts
hold the same scenario, each walks and kicks/drifts its own slice of the
sorted particles (gcs_set_step_range), and the slices of the position and
velocity arrays are exchanged after every step (the all-gather of a
multi-GPU job, here device-to-device copies through gcs_device_array, or -
in the two-process test - a gloo all-gather through host memory between
two processes).  Both slices must then hold exactly the single-context
state."""
import os
import socket

import pytest

from conftest import small_collision

pytestmark = pytest.mark.gpu


def _params(gcs):
    return gcs.reference_params(theta=0.5, epsilon_sq=0.05 ** 2, dt=0.005, leaf_size=4, walk_batch=64,
                                bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=1)


@pytest.mark.parametrize("width,graphs", [(32, False), (64, False), (32, True)])
def test_two_slices_equal_one_context(gcs_mod, width, graphs):
    import bench
    import torch
    gcs = gcs_mod
    stars = small_collision(3000, 700, 300, seed=41)  # 8,000 particles
    n = len(stars)
    p = _params(gcs)
    length, slices = bench.shard_slices(n, 2, 256)
    s = torch.cuda.Stream()
    with gcs.Context(2 * length) as a, gcs.Context(2 * length) as b, gcs.Context(n) as whole:
        for ctx, (first, count) in ((a, slices[0]), (b, slices[1])):
            ctx.set_stream(s.cuda_stream)
            ctx.set_segments([n])
            ctx.set_group_width(width)
            ctx.upload(stars)
            ctx.set_step_range(first, count)
            ctx.set_graphs(graphs)
        whole.set_stream(s.cuda_stream)
        whole.set_group_width(width)
        whole.upload(stars)
        with torch.cuda.stream(s):
            for _ in range(4):
                a.step(p)
                b.step(p)
                whole.step(p)
                for which in (gcs.BUF_POS, gcs.BUF_VEL):
                    ta = a.device_tensor(which, torch)
                    tb = b.device_tensor(which, torch)
                    f1, c1 = slices[1]
                    ta[f1:f1 + c1].copy_(tb[f1:f1 + c1])
                    tb[:slices[0][1]].copy_(ta[:slices[0][1]])
        s.synchronize()
        ref = whole.download().tobytes()
        assert a.download().tobytes() == ref
        assert b.download().tobytes() == ref
        assert a.device_status() == 0 and b.device_status() == 0


def test_step_range_bounds_are_checked(gcs_mod):
    gcs = gcs_mod
    stars = small_collision(512, 128, 64, seed=42)
    n = len(stars)
    with gcs.Context(n) as ctx:
        ctx.upload(stars)
        with pytest.raises(gcs.GcsError):
            ctx.set_step_range(17, 64)          # not a group start
        with pytest.raises(gcs.GcsError):
            ctx.set_step_range(0, n + 32)       # past the particles
        with pytest.raises(gcs.GcsError):
            ctx.set_step_range(64, n - 64)      # splits a partitioned super-group of 256
        ctx.set_walk_frontier(False)
        ctx.set_step_range(64, n - 64)          # plain groups: a group start is enough
        with pytest.raises(gcs.GcsError):
            ctx.set_walk_frontier(True)         # would partition across the range's start
        ctx.set_step_range(256, n - 256)        # to the end, on a super-group start: fine
        ctx.set_walk_frontier(True)
        with pytest.raises(gcs.GcsError):
            ctx.set_group_width(48)             # 256 is not a multiple of 48
        ctx.set_group_width(16)
        ctx.set_step_range(0, -1)               # every particle again
        assert ctx.device_array(gcs.BUF_POS) != ctx.device_array(gcs.BUF_VEL)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _slice_rank(rank, world, port, steps, out):
    """One process of the sharded step: its own context on the GPU, its slice
    stepped, the position and velocity slices all-gathered with gloo through
    host memory after every step (no kernel waits on the other process)."""
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import bench
        import gcs
        stars = small_collision(3000, 700, 300, seed=41)  # 8,000 particles
        n = len(stars)
        length, slices = bench.shard_slices(n, world, 256)
        first, count = slices[rank]
        with gcs.Context(world * length) as ctx:
            ctx.set_segments([n])
            ctx.upload(stars)
            ctx.set_step_range(first, count)
            for _ in range(steps):
                ctx.step(_params(gcs))
                for which in (gcs.BUF_POS, gcs.BUF_VEL):
                    dev = ctx.device_tensor(which, torch, rows=world * length)
                    host = dev.cpu()
                    bench.allgather_slices(dist, host, length, rank)
                    dev[:n].copy_(host[:n])
                torch.cuda.synchronize()
            out[rank] = (ctx.download().tobytes(), ctx.device_status())
    finally:
        dist.destroy_process_group()


def test_two_processes_over_gloo_equal_one_context(gcs_mod):
    """Two processes, each with its own context on its slice of one scenario,
    exchange their slices through gloo between steps; after three steps both
    hold the single-context state byte for byte."""
    import torch.multiprocessing as mp
    gcs = gcs_mod
    steps, world = 3, 2
    stars = small_collision(3000, 700, 300, seed=41)
    with gcs.Context(len(stars)) as whole:
        whole.upload(stars)
        for _ in range(steps):
            whole.step(_params(gcs))
        ref = whole.download().tobytes()
        assert whole.device_status() == 0
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_slice_rank, args=(world, _free_port(), steps, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        got, status = res[r]
        assert status == 0
        assert got == ref, "rank %d differs from the single-context state" % r
