"""Parity at the benchmark's full size: the 1,048,576-particle two-galaxy
collision (theta 0.5, eps 0.02, leaf 4, FP64 centre-of-mass sums, bounds on the
device), one step's stages through the C ABI against the oracle.

Bit-exact over every particle and node: Morton keys, the stable permutation,
the tree topology, node masses, widths, boxes and FP64-sum centres of mass.
Accelerations on a seeded sample of 16,384 targets (the oracle walks only
those): within 1e-5 relative at the 99.9th percentile (1e-4 maximum).
Size-independent properties over all particles: the keys are sorted, the
permutation is one, the root holds every particle's mass and box, and the
step keeps every particle's mass and type.  The 4,194,304-particle 1:3 pair,
the largest single-GPU scenario, gets the same stage checks."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_one_million_particles_match_oracle(gcs_mod, oracle_mod):
    gcs, oracle = gcs_mod, oracle_mod
    stars = gcs.collision_equal(384000, 96000, 44288, seed=0)
    n = len(stars)
    assert n == 1048576
    p = gcs.reference_params(theta=0.5, epsilon_sq=0.02 ** 2, dt=0.0025, leaf_size=4, walk_batch=64,
                             bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=1)
    with gcs.Context(n) as ctx:
        ctx.upload(stars)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        keys = ctx.read(gcs.BUF_KEYS)
        idx = ctx.read(gcs.BUF_INDEX)
        nodes = ctx.read(gcs.BUF_NODES)
        bd = ctx.read(gcs.BUF_BUILD)
        sp = ctx.read(gcs.BUF_POS)
        acc = ctx.read(gcs.BUF_ACCEL)
        assert ctx.device_status() == 0
        ctx.run_stages(p, gcs.STAGE_INTEGRATE, gcs.STAGE_INTEGRATE)
        after = ctx.download()

    # encode + sort
    pos, _ = gcs.pos_vel_from_stars(stars)
    lo, hi = oracle.bounds(pos)
    ks, ix = oracle.sort(oracle.encode(pos, lo, hi))
    np.testing.assert_array_equal(keys, ks)
    np.testing.assert_array_equal(idx, ix)
    assert np.all(np.diff(keys.astype(np.uint64)) >= 0)
    assert np.array_equal(np.sort(idx), np.arange(n, dtype=idx.dtype))
    np.testing.assert_array_equal(sp, pos[ix])

    # build
    cl, cr, re, par, _ = oracle.build(ks)
    np.testing.assert_array_equal(nodes["child_left"], cl)
    np.testing.assert_array_equal(nodes["child_right"], cr)
    np.testing.assert_array_equal(nodes["range_end"], re)
    np.testing.assert_array_equal(bd["parent"], par)

    # aggregate
    ref, box = oracle.aggregate(sp, cl, cr, re, com_fp64=True)
    for f in ("mass", "width", "com_x", "com_y", "com_z"):
        np.testing.assert_array_equal(nodes[f], ref[f], err_msg=f)
    np.testing.assert_array_equal(np.stack([bd["min_x"], bd["min_y"], bd["min_z"]], 1), box[:, :3])
    np.testing.assert_array_equal(np.stack([bd["max_x"], bd["max_y"], bd["max_z"]], 1), box[:, 3:])
    assert np.isclose(float(nodes["mass"][0]), float(sp[:, 3].astype(np.float64).sum()), rtol=1e-5)
    assert bd["min_x"][0] == sp[:, 0].min() and bd["max_z"][0] == sp[:, 2].max()

    # walk on a sample of targets
    targets = np.sort(np.random.default_rng(20).choice(n, 16384, replace=False))
    ref_acc, cnt = oracle.walk_targets(sp, nodes, p.G, p.epsilon_sq, p.theta, p.leaf_size, targets)
    a = acc[targets, :3]
    scale = np.median(np.linalg.norm(ref_acc[:, :3], axis=1))
    e = rel_err(a, ref_acc[:, :3], floor=1e-3 * scale)
    assert np.percentile(e, 99.9) <= 1e-5 and e.max() <= 1e-4, (np.percentile(e, 99.9), e.max())
    assert cnt[:, 0].sum() > 1000 * len(targets)  # ~1,400 terms per target at theta 0.5

    # integrate keeps every particle (same masses and types, in the new order)
    assert len(after) == n
    np.testing.assert_array_equal(np.sort(after["mass"]), np.sort(stars["mass"]))
    assert np.array_equal(np.bincount(after["type"], minlength=3), np.bincount(stars["type"], minlength=3))


def test_four_million_particle_pair_matches_oracle(gcs_mod, oracle_mod):
    """The largest single-GPU scenario: 4,194,304 particles, a 1:3 mass-ratio
    pair (impact 8, relative speed 0.6, inclination 30 degrees), theta 0.5,
    eps 0.01, leaf 4.  Keys, permutation, topology, node values and boxes
    bit-exact; accelerations of 4,096 seeded targets within 1e-5 (99.9th
    percentile); then two steps through the host step keep every particle."""
    gcs, oracle = gcs_mod, oracle_mod
    stars = gcs.collision_pair(4194304, 1.0 / 3.0, 8.0, 0.6, 30.0, 0)
    n = len(stars)
    assert n == 4194304
    p = gcs.reference_params(theta=0.5, epsilon_sq=0.01 ** 2, dt=0.002, leaf_size=4, walk_batch=64,
                             bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=1)
    with gcs.Context(n) as ctx:
        ctx.upload(stars)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        keys = ctx.read(gcs.BUF_KEYS)
        idx = ctx.read(gcs.BUF_INDEX)
        nodes = ctx.read(gcs.BUF_NODES)
        bd = ctx.read(gcs.BUF_BUILD)
        sp = ctx.read(gcs.BUF_POS)
        acc = ctx.read(gcs.BUF_ACCEL)
        assert ctx.device_status() == 0
        ctx.upload(stars)
        out = np.zeros(n, dtype=gcs.STAR_DTYPE)
        for _ in range(2):
            ctx.step_host(p, out)
        assert ctx.device_status() == 0

    pos, _ = gcs.pos_vel_from_stars(stars)
    lo, hi = oracle.bounds(pos)
    ks, ix = oracle.sort(oracle.encode(pos, lo, hi))
    np.testing.assert_array_equal(keys, ks)
    np.testing.assert_array_equal(idx, ix)
    np.testing.assert_array_equal(sp, pos[ix])
    cl, cr, re, par, _ = oracle.build(ks)
    np.testing.assert_array_equal(nodes["child_left"], cl)
    np.testing.assert_array_equal(nodes["child_right"], cr)
    np.testing.assert_array_equal(nodes["range_end"], re)
    np.testing.assert_array_equal(bd["parent"], par)
    ref, box = oracle.aggregate(sp, cl, cr, re, com_fp64=True)
    for f in ("mass", "width", "com_x", "com_y", "com_z"):
        np.testing.assert_array_equal(nodes[f], ref[f], err_msg=f)
    np.testing.assert_array_equal(np.stack([bd["min_x"], bd["min_y"], bd["min_z"]], 1), box[:, :3])
    np.testing.assert_array_equal(np.stack([bd["max_x"], bd["max_y"], bd["max_z"]], 1), box[:, 3:])

    targets = np.sort(np.random.default_rng(21).choice(n, 4096, replace=False))
    ref_acc, cnt = oracle.walk_targets(sp, nodes, p.G, p.epsilon_sq, p.theta, p.leaf_size, targets)
    scale = np.median(np.linalg.norm(ref_acc[:, :3], axis=1))
    e = rel_err(acc[targets, :3], ref_acc[:, :3], floor=1e-3 * scale)
    assert np.percentile(e, 99.9) <= 1e-5 and e.max() <= 1e-4, (np.percentile(e, 99.9), e.max())

    assert len(out) == n
    np.testing.assert_array_equal(np.sort(out["mass"]), np.sort(stars["mass"]))
    assert np.array_equal(np.bincount(out["type"], minlength=3), np.bincount(stars["type"], minlength=3))
    assert np.all(np.isfinite(out["x"])) and np.all(np.isfinite(out["vx"]))
