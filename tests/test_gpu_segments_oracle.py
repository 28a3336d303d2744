"""Batched segments checked directly against the oracle, segment by segment.

A mix like the batched workload's: twelve independent scenarios of very
uneven size (1 to 20,000 particles; sizes that are not multiples of the
64-target walk groups, so groups and super-groups end at every segment
edge), stepped as segments of one context.  Each segment is compared with
the oracle run on that segment alone: Morton keys (per-segment device
bounds), permutation, tree topology, node masses, widths, boxes and centres
of mass bit-exact (FP32 and FP64-sum centres of mass), accelerations within
the walk tolerance, and the total monopole and particle term counts equal to
the oracle's.  The solo engine path is pinned to the oracle elsewhere; this
pins the batched path without going through it.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 31, 33, 65, 257, 1000, 4097, 9000, 12000, 20000]


def _mix(gcs):
    parts = []
    for k, n in enumerate(SIZES):
        q = 0.2 + 0.8 * ((k * 37) % 11) / 10.0
        st = gcs.collision_pair(max(n, 64), q, 1.5 * k, 0.3 + 0.04 * k, 7.5 * k, seed=100 + k)
        parts.append(st[:n].copy())
    return parts


def _local_nodes(nodes, off, k, c, ni_all):
    """Segment k's internal nodes renumbered as the oracle numbers a lone
    scenario: nodes 0..c-2, particle j as c-1+j, range ends local."""
    seg = nodes[off - k: off - k + c - 1].copy()
    for f in ("child_left", "child_right"):
        v = seg[f].astype(np.int64)
        leaf = v >= ni_all
        seg[f] = np.where(leaf, v - ni_all - off + (c - 1), v - (off - k)).astype(np.int32)
    seg["range_end"] = (seg["range_end"].astype(np.int64) - off).astype(np.int32)
    return seg


@pytest.mark.parametrize("com_fp64,width,leaf", [(1, 64, 4), (0, 32, 1), (1, 48, 16)])
def test_mixed_segments_match_oracle_per_segment(gcs_mod, oracle_mod, com_fp64, width, leaf):
    gcs = gcs_mod
    parts = _mix(gcs)
    counts = [len(x) for x in parts]
    n = sum(counts)
    p = gcs.reference_params(bounds_mode=gcs.BOUNDS_DEVICE, theta=0.5, epsilon_sq=0.02 ** 2, dt=0.0025,
                             leaf_size=leaf, walk_batch=64, com_fp64=com_fp64, with_potential=1)
    with gcs.Context(n, max_segments=len(counts)) as ctx:
        ctx.set_segments(counts)
        ctx.set_group_width(width)
        ctx.upload(np.concatenate(parts))
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_WALK)
        keys = ctx.read(gcs.BUF_KEYS)
        index = ctx.read(gcs.BUF_INDEX)
        nodes = ctx.read(gcs.BUF_NODES)
        bd = ctx.read(gcs.BUF_BUILD)
        sp = ctx.read(gcs.BUF_POS)
        acc = ctx.read(gcs.BUF_ACCEL)
        total = ctx.count_interactions(p)
        assert ctx.device_status() == 0
    ni_all = n - len(counts)
    want_mono = want_part = 0
    off = 0
    for k, (c, part) in enumerate(zip(counts, parts)):
        pos, _ = gcs.pos_vel_from_stars(part)
        lo, hi = oracle_mod.bounds(pos)
        sk, idx = oracle_mod.sort(oracle_mod.encode(pos, lo, hi))
        np.testing.assert_array_equal(keys[off:off + c], sk, err_msg="keys of segment %d" % k)
        np.testing.assert_array_equal(index[off:off + c].astype(np.int64) - off, idx, err_msg="order %d" % k)
        ps = np.ascontiguousarray(pos[idx])
        np.testing.assert_array_equal(sp[off:off + c], ps, err_msg="sorted positions %d" % k)
        if c >= 2:
            cl, cr, re, par, _ = oracle_mod.build(sk)
            loc = _local_nodes(nodes, off, k, c, ni_all)
            np.testing.assert_array_equal(loc["child_left"], cl, err_msg="left children %d" % k)
            np.testing.assert_array_equal(loc["child_right"], cr, err_msg="right children %d" % k)
            np.testing.assert_array_equal(loc["range_end"], re, err_msg="ranges %d" % k)
            ref, box = oracle_mod.aggregate(ps, cl, cr, re, com_fp64=bool(com_fp64))
            for f in ("mass", "width", "com_x", "com_y", "com_z"):
                np.testing.assert_array_equal(loc[f], ref[f], err_msg="%s of segment %d" % (f, k))
            b = bd[off - k: off - k + c - 1]
            np.testing.assert_array_equal(np.stack([b["min_x"], b["min_y"], b["min_z"]], 1), box[:, :3])
            np.testing.assert_array_equal(np.stack([b["max_x"], b["max_y"], b["max_z"]], 1), box[:, 3:])
            racc, cnt = oracle_mod.walk(ps, ref, p.G, p.epsilon_sq, p.theta, leaf, counts=True)
            want_mono += int(cnt[:, 0].sum())
            want_part += int(cnt[:, 1].sum())
            scale = np.median(np.linalg.norm(racc[:, :3], axis=1))
            e = rel_err(acc[off:off + c, :3], racc[:, :3], floor=1e-3 * scale)
            assert np.percentile(e, 99.9) <= 1e-5 and e.max() <= 1e-4, (k, c, np.percentile(e, 99.9), e.max())
            np.testing.assert_allclose(acc[off:off + c, 3], racc[:, 3], rtol=1e-5, atol=1e-6 * abs(racc[:, 3]).max())
        else:
            assert np.all(acc[off:off + c] == 0.0)
        off += c
    assert total == (want_mono, want_part)
