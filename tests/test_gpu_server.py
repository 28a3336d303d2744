"""Serving: relayout keeps resident state, and the continuous-batching server
gives every scenario exactly the Stars (and simulation.bin frames) it gets
when stepped alone, however the scenarios arrive, queue and overlap."""
import os

import numpy as np
import pytest

from conftest import small_collision

pytestmark = pytest.mark.gpu


def _params(gcs, **kw):
    p = gcs.reference_params(bounds_mode=gcs.BOUNDS_DEVICE, theta=0.5, epsilon_sq=0.05 ** 2, dt=0.005,
                             leaf_size=8)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _solo(gcs, stars, p, steps, playback=False):
    with gcs.Context(len(stars)) as ctx:
        ctx.set_segments([len(stars)])
        ctx.upload(stars)
        for _ in range(steps):
            ctx.step(p)
        out = ctx.download()
        pb = ctx.download_playback() if playback else None
        assert ctx.device_status() == 0
    return out, pb


def _scenarios(gcs, k, seed0=10):
    rng = np.random.default_rng(seed0)
    out = []
    for i in range(k):
        n_total = int(rng.integers(1500, 9000))
        q = float(rng.uniform(0.2, 1.0))
        st = gcs.collision_pair(n_total, q, float(rng.uniform(0, 15)), float(rng.uniform(0.3, 0.8)),
                                float(rng.uniform(0, 90)), seed0 + i)
        out.append((st, int(rng.integers(2, 9))))
    return out


def test_relayout_keeps_state(gcs_mod):
    gcs = gcs_mod
    a = small_collision(400, 100, 50, seed=1)
    b = small_collision(300, 60, 40, seed=2)
    c = small_collision(500, 90, 30, seed=3)
    d = small_collision(200, 50, 20, seed=4)
    p = _params(gcs)
    parts = [a, b, c]
    cap = sum(len(x) for x in (a, b, c, d))
    with gcs.Context(cap, max_segments=4) as ctx:
        ctx.set_segments([len(x) for x in parts])
        ctx.upload(np.concatenate(parts))
        for _ in range(2):
            ctx.step(p)
        # b leaves, d arrives between c and a; c and a move on the device
        ctx.relayout([len(c), len(d), len(a)], [2, -1, 0])
        ctx.upload(d, offset=ctx.segment_offset(1))
        for _ in range(3):
            ctx.step(p)
        got = ctx.download()
        assert ctx.device_status() == 0
        # in place: the last segment leaves, nothing moves
        ctx.relayout([len(c), len(d)], [0, 1])
        ctx.step(p)
        got2 = ctx.download()
    offs = np.cumsum([0, len(c), len(d), len(a)])
    for part, steps, k in ((c, 5, 0), (d, 3, 1), (a, 5, 2)):
        ref, _ = _solo(gcs, part, p, steps)
        assert got[offs[k]:offs[k + 1]].tobytes() == ref.tobytes()
    for part, steps, k in ((c, 6, 0), (d, 4, 1)):
        ref, _ = _solo(gcs, part, p, steps)
        assert got2[offs[k]:offs[k + 1]].tobytes() == ref.tobytes()


def test_relayout_rejects_bad_layouts(gcs_mod):
    gcs = gcs_mod
    a = small_collision(100, 20, 10, seed=1)
    with gcs.Context(2 * len(a), max_segments=2) as ctx:
        ctx.set_segments([len(a), len(a)])
        ctx.upload(np.concatenate([a, a]))
        with pytest.raises(gcs.GcsError):
            ctx.relayout([len(a) + 1], [0])        # a kept segment changes its count
        with pytest.raises(gcs.GcsError):
            ctx.relayout([len(a), len(a)], [0, 0])  # one segment kept twice
        with pytest.raises(gcs.GcsError):
            ctx.relayout([len(a)], [5])             # no such segment


def test_server_results_equal_solo(gcs_mod, tmp_path):
    """Staggered arrivals through a 3-slot server: every final state and every
    simulation.bin frame is byte-identical to the scenario stepped alone."""
    gcs = gcs_mod
    p = _params(gcs)
    scen = _scenarios(gcs, 7)
    total = sum(len(s) for s, _ in scen)
    frame_every = 3
    with gcs.Server(p, max_particles=total, max_segments=3, hbm_budget_bytes=1e12) as srv:
        srv.set_output(str(tmp_path), frame_every)
        arrivals = {0: [0, 1], 2: [2, 3, 4], 3: [5], 7: [6]}
        done = {}
        peak_resident = 0
        for t in range(200):
            for i in arrivals.get(t, []):
                srv.submit(i, scen[i][0], scen[i][1])
            resident, particles, admitted, retired = srv.tick()
            peak_resident = max(peak_resident, resident)
            assert resident <= 3
            while True:
                r = srv.pop()
                if r is None:
                    break
                info, stars = r
                assert info.status == 0 and info.latency_ms >= info.queued_ms >= 0
                done[int(info.id)] = stars
            if len(done) == len(scen):
                break
        assert len(done) == len(scen)
        assert peak_resident == 3   # scenarios overlapped on the device
        assert srv.counts() == (0, 0, 0)
    for i, (st, steps) in enumerate(scen):
        ref, pb = _solo(gcs, st, p, steps, playback=True)
        assert done[i].tobytes() == ref.tobytes(), "scenario %d differs from its solo run" % i
        frames = gcs.read_playback(os.path.join(str(tmp_path), "%d.bin" % i), len(st))
        assert len(frames) == steps // frame_every + (1 if steps % frame_every else 0)
        assert frames[-1].tobytes() == pb.tobytes()
        if steps > frame_every:
            _, pb3 = _solo(gcs, st, p, frame_every, playback=True)
            assert frames[0].tobytes() == pb3.tobytes()


def test_server_budget_and_capacity(gcs_mod):
    gcs = gcs_mod
    p = _params(gcs)
    a = small_collision(400, 100, 50, seed=1)
    with gcs.Context(1000, max_segments=4) as probe:
        assert probe.device_bytes == gcs.context_bytes(1000, 4)
    budget = gcs.context_bytes(3 * len(a) // 2, 4)
    with gcs.Server(p, max_particles=10 * len(a), max_segments=4, hbm_budget_bytes=budget) as srv:
        cap = srv.capacity
        assert cap == 3 * len(a) // 2 or gcs.context_bytes(cap + 1, 4) > budget
        assert len(a) <= cap < 2 * len(a)
        assert srv.device_bytes <= budget
        with pytest.raises(gcs.GcsError):
            srv.submit(99, np.concatenate([a] * 10), 1)
        srv.submit(1, a, 2)
        srv.submit(2, a, 2)     # does not fit beside the first: waits
        res = srv.tick()
        assert res[0] == 1 and res[1] == len(a)
        assert srv.counts()[0] == 1
        ids = []
        for _ in range(10):
            srv.tick()
            while (r := srv.pop(with_stars=False)) is not None:
                ids.append(int(r[0].id))
            if len(ids) == 2:
                break
        assert ids == [1, 2]
