"""GPU parity: every stage of the CUDA path against the oracle on the same
seeded inputs, called through the C ABI.

Bars: bit-exact for keys, permutation, topology, bounds, masses, widths and
the integrate step (same inputs); accelerations within 1e-5 relative
(FP32 reassociation and rsqrtf vs IEEE 1/sqrt only), measured per particle
as |a - a_ref| / max(|a_ref|, 1e-3 * median |a_ref|), required at the 99.9th
percentile, with 1e-4 as the per-particle maximum.  At theta = 0 (a direct
sum over every particle) the FP32 rounding of the sum itself, in any order,
is above 1e-5 for the particles with the most cancellation; there the engine
and the oracle are both compared with an FP64 direct sum and the engine must
be at least as close as the oracle."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err, small_collision

pytestmark = pytest.mark.gpu

TOL_ACC = 1e-5
TOL_ACC_MAX = 1e-4


def _acc_err(a, ref):
    scale = np.median(np.linalg.norm(ref, axis=1))
    return rel_err(a, ref, floor=1e-3 * scale)


def _assert_acc(a, ref, what=""):
    e = _acc_err(a, ref)
    assert np.percentile(e, 99.9) <= TOL_ACC, (what, np.percentile(e, 99.9))
    assert e.max() <= TOL_ACC_MAX, (what, e.max())


@pytest.fixture(scope="module")
def stars():
    return small_collision(2048, 512, 256, seed=11)  # 5632 particles


def _params(gcs, **kw):
    p = gcs.reference_params(bounds_mode=gcs.BOUNDS_DEVICE, theta=0.5, epsilon_sq=0.05 ** 2, dt=0.005,
                             leaf_size=1)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _ctx(gcs, stars, segments=None):
    n = len(stars)
    ctx = gcs.Context(n, max_segments=len(segments) if segments else 1)
    ctx.set_segments(segments or [n])
    ctx.upload(stars)
    return ctx


def test_bounds_and_encode_bitexact(gcs_mod, oracle_mod, stars):
    gcs = gcs_mod
    pos, _ = gcs.pos_vel_from_stars(stars)
    with _ctx(gcs, stars) as ctx:
        p = _params(gcs)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_ENCODE)
        lo, hi = oracle_mod.bounds(pos)
        np.testing.assert_array_equal(ctx.read(gcs.BUF_BOUNDS)[0], [lo, hi])
        np.testing.assert_array_equal(ctx.read(gcs.BUF_KEYS_UNSORTED), oracle_mod.encode(pos, lo, hi))
        # caller bounds (the reference API), including particles outside the cube
        p = _params(gcs, bounds_mode=gcs.BOUNDS_CALLER, global_min=-30.0, global_max=20.0)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_ENCODE)
        np.testing.assert_array_equal(ctx.read(gcs.BUF_KEYS_UNSORTED),
                                      oracle_mod.encode(pos, np.float32(-30.0), np.float32(20.0)))
        assert ctx.device_status() == 0


@pytest.mark.parametrize("n", [1, 2, 3, 4095, 4096, 4097, 70001])
def test_sort_bitexact(gcs_mod, oracle_mod, n):
    gcs = gcs_mod
    st = small_collision(max(n // 2, 1), 0, 0, seed=n)[:n]
    if len(st) < n:
        st = np.resize(st, n)
    rng = np.random.default_rng(n)
    if n > 10:  # force duplicate keys
        st["x"][: n // 3] = st["x"][0]
        st["y"][: n // 3] = st["y"][0]
        st["z"][: n // 3] = st["z"][0]
    st["x"] += rng.normal(0, 1e-3, n).astype(np.float32) * (rng.random(n) < 0.5)
    pos, _ = gcs.pos_vel_from_stars(st)
    with _ctx(gcs, st) as ctx:
        p = _params(gcs)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_SORT)
        lo, hi = oracle_mod.bounds(pos)
        sk, idx = oracle_mod.sort(oracle_mod.encode(pos, lo, hi))
        np.testing.assert_array_equal(ctx.read(gcs.BUF_KEYS), sk)
        np.testing.assert_array_equal(ctx.read(gcs.BUF_INDEX), idx)
        assert ctx.device_status() == 0


def test_build_topology_bitexact(gcs_mod, oracle_mod, stars):
    gcs = gcs_mod
    pos, _ = gcs.pos_vel_from_stars(stars)
    n = len(stars)
    with _ctx(gcs, stars) as ctx:
        ctx.run_stages(_params(gcs), gcs.STAGE_BOUNDS, gcs.STAGE_BUILD)
        lo, hi = oracle_mod.bounds(pos)
        sk, _ = oracle_mod.sort(oracle_mod.encode(pos, lo, hi))
        cl, cr, re, par, lp = oracle_mod.build(sk)
        nodes = ctx.read(gcs.BUF_NODES)
        np.testing.assert_array_equal(nodes["child_left"], cl)
        np.testing.assert_array_equal(nodes["child_right"], cr)
        np.testing.assert_array_equal(nodes["range_end"], re)
        np.testing.assert_array_equal(ctx.read(gcs.BUF_BUILD)["parent"], par)
        np.testing.assert_array_equal(ctx.read(gcs.BUF_LEAF_PARENT), lp)
        assert ctx.n_internal == n - 1
        assert ctx.device_status() == 0


@pytest.mark.parametrize("com_fp64", [0, 1])
def test_aggregate(gcs_mod, oracle_mod, stars, com_fp64):
    gcs = gcs_mod
    with _ctx(gcs, stars) as ctx:
        ctx.run_stages(_params(gcs, com_fp64=com_fp64), gcs.STAGE_BOUNDS, gcs.STAGE_AGGREGATE)
        sp = ctx.read(gcs.BUF_POS)
        nodes = ctx.read(gcs.BUF_NODES)
        bd = ctx.read(gcs.BUF_BUILD)
        ref, box = oracle_mod.aggregate(sp, nodes["child_left"], nodes["child_right"], nodes["range_end"],
                                        com_fp64=bool(com_fp64))
        np.testing.assert_array_equal(nodes["mass"], ref["mass"])
        np.testing.assert_array_equal(nodes["width"], ref["width"])
        np.testing.assert_array_equal(np.stack([bd["min_x"], bd["min_y"], bd["min_z"]], 1), box[:, :3])
        np.testing.assert_array_equal(np.stack([bd["max_x"], bd["max_y"], bd["max_z"]], 1), box[:, 3:])
        for a in ("com_x", "com_y", "com_z"):
            np.testing.assert_array_equal(nodes[a], ref[a], err_msg=a)


@pytest.mark.parametrize("theta,leaf", [(1.0, 1), (0.5, 1), (0.5, 8), (0.5, 32), (0.7, 16), (0.0, 4)])
def test_walk_matches_oracle(gcs_mod, oracle_mod, stars, theta, leaf):
    gcs = gcs_mod
    with _ctx(gcs, stars) as ctx:
        p = _params(gcs, theta=theta, leaf_size=leaf, with_potential=1)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        sp = ctx.read(gcs.BUF_POS)
        nodes = ctx.read(gcs.BUF_NODES)
        acc = ctx.read(gcs.BUF_ACCEL)
        ref = oracle_mod.walk(sp, nodes, p.G, p.epsilon_sq, theta, leaf)
        if theta > 0:
            _assert_acc(acc[:, :3], ref[:, :3], "theta=%s L=%s" % (theta, leaf))
        else:
            # theta = 0 is a direct sum over every particle: its FP32 rounding
            # (in the oracle's order or any other) exceeds 1e-5 for the
            # particles with the most cancellation, so both sums are held to
            # an FP64 direct sum and the engine must be at least as close
            exact = ctx.direct_fp64(p, np.arange(len(sp)))
            scale = np.median(np.linalg.norm(exact, axis=1))
            e_gpu = rel_err(acc[:, :3], exact, floor=1e-3 * scale)
            e_ref = rel_err(ref[:, :3], exact, floor=1e-3 * scale)
            assert np.percentile(e_gpu, 99.9) <= max(TOL_ACC, np.percentile(e_ref, 99.9))
            assert e_gpu.max() <= TOL_ACC_MAX
            assert _acc_err(acc[:, :3], ref[:, :3]).max() <= TOL_ACC_MAX
        np.testing.assert_allclose(acc[:, 3], ref[:, 3], rtol=1e-5)
        assert ctx.device_status() == 0


@pytest.mark.parametrize("batch", [1, 4, 32, 33, 64])
def test_walk_batch_sizes_agree(gcs_mod, stars, batch):
    gcs = gcs_mod
    with _ctx(gcs, stars) as ctx:
        ctx.run_stages(_params(gcs, walk_batch=1, leaf_size=8), gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        a1 = ctx.read(gcs.BUF_ACCEL)
        ctx.run_stages(_params(gcs, walk_batch=batch, leaf_size=8), gcs.STAGE_WALK, gcs.STAGE_WALK)
        a2 = ctx.read(gcs.BUF_ACCEL)
        _assert_acc(a2[:, :3], a1[:, :3])


@pytest.mark.parametrize("width,batch,theta,leaf", [(64, 64, 0.5, 4), (64, 32, 0.5, 1), (64, 64, 1.0, 1),
                                                   (48, 64, 0.7, 8), (40, 16, 0.5, 32)])
def test_wide_groups_match_oracle(gcs_mod, oracle_mod, stars, width, batch, theta, leaf):
    """Groups wider than 32 hold two targets per lane; every target still
    takes exactly its own terms: accelerations within the walk tolerance of
    the oracle and the same number of monopole and particle terms as the
    oracle's per-target walk."""
    gcs = gcs_mod
    with _ctx(gcs, stars) as ctx:
        ctx.set_group_width(width)
        assert ctx.group_width == width
        p = _params(gcs, theta=theta, leaf_size=leaf, walk_batch=batch, with_potential=1)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        sp = ctx.read(gcs.BUF_POS)
        nodes = ctx.read(gcs.BUF_NODES)
        acc = ctx.read(gcs.BUF_ACCEL)
        ref, cnt = oracle_mod.walk(sp, nodes, p.G, p.epsilon_sq, theta, leaf, counts=True)
        _assert_acc(acc[:, :3], ref[:, :3], "width=%d batch=%d theta=%s L=%d" % (width, batch, theta, leaf))
        np.testing.assert_allclose(acc[:, 3], ref[:, 3], rtol=1e-5)
        n_mono, n_part = ctx.count_interactions(p)
        assert (n_mono, n_part) == (int(cnt[:, 0].sum()), int(cnt[:, 1].sum()))
        assert ctx.device_status() == 0


@pytest.mark.parametrize("width,theta,leaf", [(32, 0.5, 4), (16, 0.5, 1), (64, 0.5, 8), (32, 0.7, 32),
                                               (48, 1.0, 1), (32, 0.3, 2)])
def test_walk_frontier_keeps_every_targets_terms(gcs_mod, oracle_mod, width, theta, leaf):
    """The super-group frontier pass (on by default) and the walk from the
    root (frontiers off) give every target exactly the oracle's terms: the
    same monopole and particle counts, accelerations and potentials within
    the walk tolerance; several super-groups of uneven size per segment."""
    gcs = gcs_mod
    st = small_collision(4096, 1024, 512, seed=31)  # 11,264 particles
    with _ctx(gcs, st) as ctx:
        ctx.set_group_width(width)
        p = _params(gcs, theta=theta, leaf_size=leaf, walk_batch=64, with_potential=1)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_AGGREGATE)
        sp = ctx.read(gcs.BUF_POS)
        ref, cnt = oracle_mod.walk(sp, ctx.read(gcs.BUF_NODES), p.G, p.epsilon_sq, theta, leaf, counts=True)
        want = (int(cnt[:, 0].sum()), int(cnt[:, 1].sum()))
        for frontier in (True, False):
            ctx.set_walk_frontier(frontier)
            ctx.run_stages(p, gcs.STAGE_WALK, gcs.STAGE_WALK)
            acc = ctx.read(gcs.BUF_ACCEL)
            _assert_acc(acc[:, :3], ref[:, :3], "frontier=%s width=%d theta=%s L=%d" % (frontier, width, theta, leaf))
            np.testing.assert_allclose(acc[:, 3], ref[:, 3], rtol=1e-5)
            assert ctx.count_interactions(p) == want, frontier
            peak, global_cap = ctx.walk_stack_peak()
            # the deepest stack a walk warp held fits the shared top plus the global bottom
            assert 0 < peak <= global_cap + 512, (frontier, peak)
            # every monopole term came from a row: full rows serve at most 32
            # lanes, other take rows and mixed rows the lanes counted for them
            lu = ctx.walk_lane_use()
            n_mono, n_part = want
            slots = 64 if width > 32 else 32  # target slots of a walk warp
            some = lu["lanes_take_partial"] + lu["lanes_mixed_accepting"]
            assert some <= n_mono <= some + slots * (lu["rows_take_list"] + lu["rows_take_full"]), lu
            assert lu["lanes_mixed_accepting"] <= lu["lanes_mixed"] <= slots * lu["rows_mixed"], lu
            assert lu["lanes_take_partial"] <= slots * lu["rows_take_partial"], lu
            assert n_part <= lu["lanes_source"], lu
            if not frontier:
                assert lu["rows_take_list"] == 0, lu
        assert ctx.device_status() == 0


def test_wide_groups_in_segments(gcs_mod, stars):
    """Two targets per lane over uneven segments (groups never straddle a
    segment): each segment's accelerations equal the segment walked alone."""
    gcs = gcs_mod
    a = small_collision(700, 170, 91, seed=21)   # 1,922 particles: not a multiple of 64
    b = small_collision(300, 64, 33, seed=22)    # 794
    p = _params(gcs, leaf_size=4, walk_batch=64)
    with _ctx(gcs, np.concatenate([a, b]), segments=[len(a), len(b)]) as both:
        both.set_group_width(64)
        both.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        acc_both = both.read(gcs.BUF_ACCEL)
        assert both.device_status() == 0
    for k, part in enumerate((a, b)):
        with _ctx(gcs, part) as solo:
            solo.set_group_width(64)
            solo.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
            off = 0 if k == 0 else len(a)
            assert np.array_equal(solo.read(gcs.BUF_ACCEL), acc_both[off:off + len(part)])


def test_group_width_and_autotune(gcs_mod, oracle_mod, stars):
    """Group width changes only the order of the sums; the autotuner returns
    settings within the caller's leaf bound whose results match the oracle."""
    gcs = gcs_mod
    with _ctx(gcs, stars) as ctx:
        p = _params(gcs, leaf_size=8)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        a32 = ctx.read(gcs.BUF_ACCEL)
        ctx.set_group_width(16)
        assert ctx.group_width == 16
        ctx.run_stages(p, gcs.STAGE_WALK, gcs.STAGE_WALK)
        _assert_acc(ctx.read(gcs.BUF_ACCEL)[:, :3], a32[:, :3], "width 16 vs 32")
        with pytest.raises(gcs.GcsError):
            ctx.set_group_width(4)
        q, ms = ctx.autotune(_params(gcs, leaf_size=8))
        assert 1 <= q.leaf_size <= 8 and q.walk_batch in (16, 32, 64) and ms > 0
        ctx.run_stages(q, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        ref = oracle_mod.walk(ctx.read(gcs.BUF_POS), ctx.read(gcs.BUF_NODES), q.G, q.epsilon_sq, q.theta,
                              q.leaf_size)
        _assert_acc(ctx.read(gcs.BUF_ACCEL)[:, :3], ref[:, :3], "autotuned")
        assert ctx.device_status() == 0


@pytest.mark.parametrize("width", [32, 64])
def test_kick_in_walk_equals_integrate_launch(gcs_mod, width):
    """A full step applies the kick/drift in the walk's epilogue; running the
    walk and the integrate stage in separate calls launches integrate_kernel.
    Both give the same bytes, over uneven segments (a 1-particle one too)."""
    gcs = gcs_mod
    a = small_collision(1500, 400, 211, seed=51)
    b = small_collision(300, 90, 17, seed=52)
    one = small_collision(64, 16, 8, seed=53)[:1]
    st = np.concatenate([a, one, b])
    segs = [len(a), 1, len(b)]
    p = _params(gcs, leaf_size=4, walk_batch=64, com_fp64=1)
    with _ctx(gcs, st, segs) as fused, _ctx(gcs, st, segs) as split:
        fused.set_group_width(width)
        split.set_group_width(width)
        for _ in range(3):
            fused.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_INTEGRATE)
            split.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
            split.run_stages(p, gcs.STAGE_INTEGRATE, gcs.STAGE_INTEGRATE)
            assert fused.download().tobytes() == split.download().tobytes()
            np.testing.assert_array_equal(fused.read(gcs.BUF_ACCEL), split.read(gcs.BUF_ACCEL))
        assert fused.device_status() == 0 and split.device_status() == 0


def test_walk_events_time_eager_and_graph_steps(gcs_mod, stars):
    """Caller events around the walk stage: recorded in eager steps and
    inside captured steps, re-pointed per step without a new capture, and
    the state stays byte-identical to steps without events."""
    import torch
    gcs = gcs_mod
    s = torch.cuda.Stream()
    p = _params(gcs, leaf_size=4, com_fp64=1)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(6)]
    for a, b in evs:
        a.record(s)
        b.record(s)
    with _ctx(gcs, stars) as plain, _ctx(gcs, stars) as timed:
        plain.set_stream(s.cuda_stream)
        timed.set_stream(s.cuda_stream)
        for k in range(2):  # eager
            timed.set_walk_events(*evs[k])
            timed.step(p)
            plain.step(p)
        plain.set_graphs(True)
        timed.set_graphs(True)
        for k in range(2, 6):  # captured once, events re-pointed each step
            timed.set_walk_events(*evs[k])
            timed.step(p)
            plain.step(p)
        torch.cuda.synchronize()
        assert timed.graph_builds == 1
        walk = [a.elapsed_time(b) for a, b in evs]
        assert all(w > 0.0 for w in walk), walk
        assert plain.download().tobytes() == timed.download().tobytes()
        timed.set_walk_events(None, None)  # presence changes: captured again
        timed.step(p)
        plain.step(p)
        assert timed.graph_builds == 2
        assert plain.download().tobytes() == timed.download().tobytes()
        assert timed.device_status() == 0


def test_graph_steps_match_eager_steps(gcs_mod, stars):
    """The captured step is the eager step: byte-identical state after
    several steps, one capture per parameter set."""
    import torch
    gcs = gcs_mod
    s = torch.cuda.Stream()
    with _ctx(gcs, stars) as eager, _ctx(gcs, stars) as graph:
        eager.set_stream(s.cuda_stream)
        graph.set_stream(s.cuda_stream)
        graph.set_graphs(True)
        p = _params(gcs, leaf_size=4, com_fp64=1)
        for _ in range(5):
            eager.step(p)
            graph.step(p)
        assert graph.graph_builds == 1
        assert eager.download().tobytes() == graph.download().tobytes()
        q = _params(gcs, leaf_size=8, com_fp64=1)
        for _ in range(3):
            eager.step(q)
            graph.step(q)
        assert graph.graph_builds == 2
        assert eager.download().tobytes() == graph.download().tobytes()
        np.testing.assert_array_equal(eager.read(gcs.BUF_ACCEL), graph.read(gcs.BUF_ACCEL))
        assert graph.device_status() == 0
    with _ctx(gcs, stars) as c:
        with pytest.raises(gcs.GcsError):  # the legacy default stream cannot be captured
            c.set_graphs(True)


def test_integrate_bitexact(gcs_mod, oracle_mod, stars):
    gcs = gcs_mod
    with _ctx(gcs, stars) as ctx:
        # large speeds so the colour map crosses both branches
        s2 = stars.copy()
        rng = np.random.default_rng(3)
        s2["vx"] = rng.uniform(-200, 200, len(s2)).astype(np.float32)
        ctx.upload(s2)
        p = _params(gcs, dt=0.01)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        x0, v0, a = ctx.read(gcs.BUF_POS), ctx.read(gcs.BUF_VEL), ctx.read(gcs.BUF_ACCEL)
        ctx.run_stages(p, gcs.STAGE_INTEGRATE, gcs.STAGE_INTEGRATE)
        x1, v1 = ctx.read(gcs.BUF_POS), ctx.read(gcs.BUF_VEL)
        xr, vr = oracle_mod.integrate(x0, v0, a, p.dt, True)
        np.testing.assert_array_equal(x1, xr)
        np.testing.assert_array_equal(v1.view(np.uint32), vr.view(np.uint32))


def test_full_step_matches_oracle_step(gcs_mod, oracle_mod, stars):
    gcs = gcs_mod
    pos, vel = gcs.pos_vel_from_stars(stars)
    for leaf in (1, 16):
        with _ctx(gcs, stars) as ctx:
            p = _params(gcs, leaf_size=leaf)
            ctx.step(p)
            out = ctx.download()
            acc = ctx.read(gcs.BUF_ACCEL)
            xr, vr, ar, _ = oracle_mod.step(pos, vel, p.G, p.epsilon_sq, p.theta, leaf, p.dt)
            sr = gcs.stars_from_pos_vel(xr, vr)
            _assert_acc(acc[:, :3], ar[:, :3], "step L=%d" % leaf)
            for f in ("mass", "type"):
                np.testing.assert_array_equal(out[f], sr[f])
            for f in ("x", "y", "z", "vx", "vy", "vz"):
                np.testing.assert_allclose(out[f], sr[f], rtol=1e-6, atol=1e-6)
            assert ctx.device_status() == 0


def test_segments_match_solo_bitwise(gcs_mod, stars):
    """Scenarios batched as segments give exactly their solo results."""
    gcs = gcs_mod
    a = stars[:1]
    b = stars[1:3]
    c = small_collision(300, 100, 77, seed=5)
    d = stars[3:3 + 4101]
    parts = [a, b, c, d]
    allst = np.concatenate(parts)
    p = _params(gcs, leaf_size=8)
    with _ctx(gcs, allst, segments=[len(x) for x in parts]) as ctx:
        for _ in range(3):
            ctx.step(p)
        batched = ctx.download()
        bacc = ctx.read(gcs.BUF_ACCEL)
        assert ctx.device_status() == 0
    off = 0
    for part in parts:
        with _ctx(gcs, part) as solo:
            for _ in range(3):
                solo.step(p)
            np.testing.assert_array_equal(solo.download().tobytes(), batched[off:off + len(part)].tobytes())
            np.testing.assert_array_equal(solo.read(gcs.BUF_ACCEL), bacc[off:off + len(part)])
        off += len(part)


def test_edge_cases(gcs_mod, oracle_mod):
    gcs = gcs_mod
    st = small_collision(64, 16, 8, seed=2)
    # one particle: no force
    with _ctx(gcs, st[:1]) as ctx:
        ctx.step(_params(gcs))
        assert np.all(ctx.read(gcs.BUF_ACCEL) == 0)
    # every particle at one point: degenerate cube, all keys equal, self exclusion
    same = st.copy()
    same["x"], same["y"], same["z"] = 1.5, 1.5, 1.5   # max == min: scale is inf, (x-min)*scale is NaN -> 0
    with _ctx(gcs, same) as ctx:
        # the FP32 pairwise formula (every node here is below the FP64 size)
        # rounds the COM of unequal masses off the point by an ulp: with
        # either setting the result must be the oracle's
        for com in (1, 0):
            p = _params(gcs, com_fp64=com)
            ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
            assert np.all(ctx.read(gcs.BUF_KEYS) == 0)
            nodes = ctx.read(gcs.BUF_NODES)
            ref_nodes, _ = oracle_mod.aggregate(ctx.read(gcs.BUF_POS), nodes["child_left"], nodes["child_right"],
                                                nodes["range_end"], com_fp64=bool(com))
            for f in ("com_x", "com_y", "com_z", "mass"):
                np.testing.assert_array_equal(nodes[f], ref_nodes[f])
            ref = oracle_mod.walk(ctx.read(gcs.BUF_POS), nodes, p.G, p.epsilon_sq, p.theta, 1)
            np.testing.assert_allclose(ctx.read(gcs.BUF_ACCEL)[:, :3], ref[:, :3], rtol=1e-5)
        assert ctx.device_status() == 0
    # two particles
    with _ctx(gcs, st[:2]) as ctx:
        p = _params(gcs)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        sp = ctx.read(gcs.BUF_POS)
        ex = oracle_mod.direct_fp64(sp, [0, 1], p.G, p.epsilon_sq)
        _assert_acc(ctx.read(gcs.BUF_ACCEL)[:, :3], ex)
    # a NaN position is reported through the device status word
    bad = st.copy()
    bad["x"][5] = np.nan
    with _ctx(gcs, bad) as ctx:
        ctx.run_stages(_params(gcs), gcs.STAGE_BOUNDS, gcs.STAGE_BOUNDS)
        assert ctx.device_status(clear=True) & gcs.DEV_NONFINITE_POSITION
        assert ctx.device_status() == 0


def test_bad_arguments_are_rejected(gcs_mod, stars):
    gcs = gcs_mod
    with _ctx(gcs, stars) as ctx:
        with pytest.raises(gcs.GcsError):
            ctx.step(_params(gcs, leaf_size=0))
        with pytest.raises(gcs.GcsError):
            ctx.step(_params(gcs, leaf_size=33))
        with pytest.raises(gcs.GcsError):
            ctx.set_segments([len(stars) + 1])
        with pytest.raises(gcs.GcsError):
            ctx.set_segments([0, len(stars)])


def test_dropin_cpp_api(gcs_mod, oracle_mod, stars):
    """The reference's C++ entry points, called by their mangled names."""
    gcs = gcs_mod
    L = gcs.lib()
    f = {}
    for name, sym, res, args in [
        ("init", "_Z9cuda_initi", C.c_bool, [C.c_int]),
        ("cleanup", "_Z12cuda_cleanupv", None, []),
        ("upload", "_Z25cuda_upload_initial_starsPK4Stari", None, [C.c_void_p, C.c_int]),
        ("step", "_Z17cuda_physics_stepP4Starifffffb", C.c_float,
         [C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_bool]),
        ("com", "_Z23cuda_get_center_of_massPfS_S_", None, [C.c_void_p] * 3),
        ("alloc", "_Z26cuda_allocate_pinned_starsPP4Stari", None, [C.c_void_p, C.c_int]),
        ("free", "_Z22cuda_free_pinned_starsP4Star", None, [C.c_void_p]),
        ("reg", "_Z17cuda_register_vboj", None, [C.c_uint]),
        ("unreg", "_Z19cuda_unregister_vbov", None, []),
    ]:
        fn = getattr(L, sym)
        fn.restype, fn.argtypes = res, args
        f[name] = fn
    n = len(stars)
    assert f["init"](n)
    try:
        f["upload"](stars.ctypes.data, n)
        pinned = C.c_void_p()
        f["alloc"](C.byref(pinned), n)
        assert pinned.value
        host = np.ctypeslib.as_array((C.c_byte * (32 * n)).from_address(pinned.value)).view(gcs.STAR_DTYPE)
        pos, vel = gcs.pos_vel_from_stars(stars)
        lo, hi = oracle_mod.bounds(pos)
        dt = f["step"](pinned, n, 1.0, 10.0, 0.01, float(lo), float(hi), False)
        assert dt == pytest.approx(0.01)
        xr, vr, ar, nodes = oracle_mod.step(pos, vel, 1.0, 10.0, 1.0, 1, 0.01, bounds_lohi=(lo, hi))
        sr = gcs.stars_from_pos_vel(xr, vr)
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            np.testing.assert_allclose(host[k], sr[k], rtol=1e-6, atol=1e-6)
        np.testing.assert_array_equal(host["mass"], sr["mass"])
        cx, cy, cz = C.c_float(), C.c_float(), C.c_float()
        f["com"](C.byref(cx), C.byref(cy), C.byref(cz))
        np.testing.assert_allclose([cx.value, cy.value, cz.value],
                                   [nodes["com_x"][0], nodes["com_y"][0], nodes["com_z"][0]], rtol=1e-5)
        # interop: stepped stars go to the headless device buffer, host untouched
        f["reg"](7)
        before = host.copy()
        f["step"](pinned, n, 1.0, 10.0, 0.01, float(lo), float(hi), True)
        np.testing.assert_array_equal(host, before)
        assert L.gcs_dropin_device_stars()
        f["unreg"]()
        f["free"](pinned)
    finally:
        f["cleanup"]()
