"""The oracle (CPU restatement of the reference path) pinned against the
reference's own code: golden vectors made by tests/golden/make_golden.py
from the reference sources, plus the properties the reference's algorithm
guarantees.  CPU only."""
import glob
import os

import numpy as np
import pytest

from conftest import rel_err, small_collision

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_morton_matches_reference_golden(oracle_mod):
    g = np.load(os.path.join(GOLDEN, "morton_ref.npz"))
    names = sorted({k[: -len("_keys")] for k in g.files if k.endswith("_keys")})
    assert names, "no golden Morton cases"
    for name in names:
        xyz = g[name + "_xyz"]
        lo, hi = g[name + "_lohi"]
        xyzm = np.concatenate([xyz, np.ones((len(xyz), 1), np.float32)], axis=1)
        keys = oracle_mod.encode(xyzm, lo, hi)
        np.testing.assert_array_equal(keys, g[name + "_keys"], err_msg=name)
    spread = [oracle_mod.lib().gcs_oracle_spread21(int(v)) for v in g["expand_in"]]
    np.testing.assert_array_equal(np.array(spread, np.uint64), g["expand_out"])


def test_morton_wrap_and_saturation(oracle_mod):
    o = oracle_mod.lib()
    # the GPU conversion saturates: negative / NaN -> 0, huge -> 2^32-1
    assert o.gcs_oracle_f2u_rz(-5.0) == 0
    assert o.gcs_oracle_f2u_rz(float("nan")) == 0
    assert o.gcs_oracle_f2u_rz(1e20) == 0xFFFFFFFF
    assert o.gcs_oracle_f2u_rz(2097151.9) == 2097151
    # a coordinate that quantises to 2^21 keeps only its low 21 bits (wraps to 0)
    lo, hi = np.float32(0.0), np.float32(1.0)
    scale = np.float32(2097151.0) / (hi - lo)
    x = np.float32(2097152.0) / scale
    while np.float32(x - lo) * scale < np.float32(2097152.0):
        x = np.nextafter(x, np.float32(2.0))
    assert o.gcs_oracle_morton(float(x), 0.0, 0.0, float(lo), float(hi)) == 0


def test_sort_is_stable_with_position_tiebreak(oracle_mod):
    rng = np.random.default_rng(0)
    keys = rng.integers(0, 50, size=5000).astype(np.uint64) << np.uint64(40)
    sk, idx = oracle_mod.sort(keys)
    np.testing.assert_array_equal(idx, np.argsort(keys, kind="stable"))
    np.testing.assert_array_equal(sk, np.sort(keys))


def _tree_invariants(cl, cr, re, par, lp, n):
    ni = n - 1
    seen_leaf = np.zeros(n, bool)
    seen_node = np.zeros(ni, bool)
    stack = [(0, 0, n - 1)]
    while stack:
        v, lo, hi = stack.pop()
        assert not seen_node[v]
        seen_node[v] = True
        assert min(v, re[v]) == lo and max(v, re[v]) == hi
        for c, side in ((cl[v], 0), (cr[v], 1)):
            if c >= ni:
                k = c - ni
                assert not seen_leaf[k] and lp[k] == v
                seen_leaf[k] = True
            else:
                assert par[c] == v
        # children partition [lo, hi]
        gl = cl[v] - ni if cl[v] >= ni else cl[v]
        split = gl if cl[v] >= ni else max(cl[v], re[cl[v]])
        left_hi = split
        right_lo = split + 1
        c = cr[v]
        r_lo = c - ni if c >= ni else min(c, re[c])
        assert r_lo == right_lo
        if cl[v] < ni:
            stack.append((cl[v], lo, left_hi))
        if cr[v] < ni:
            stack.append((cr[v], right_lo, hi))
    assert seen_leaf.all() and seen_node.all()
    assert par[0] == -1


@pytest.mark.parametrize("n", [2, 3, 5, 64, 1000])
def test_karras_tree_invariants(oracle_mod, n):
    rng = np.random.default_rng(n)
    pts = rng.uniform(-1, 1, size=(n, 4)).astype(np.float32)
    pts[:, 3] = 1.0
    lo, hi = oracle_mod.bounds(pts)
    sk, _ = oracle_mod.sort(oracle_mod.encode(pts, lo, hi))
    _tree_invariants(*oracle_mod.build(sk), n)


def test_karras_tree_with_duplicate_keys(oracle_mod):
    keys = np.array([5, 5, 5, 5, 9, 9, 12, 12, 12, 40], np.uint64)
    _tree_invariants(*oracle_mod.build(keys), len(keys))
    keys = np.zeros(17, np.uint64)  # every key equal: the position bits decide
    _tree_invariants(*oracle_mod.build(keys), len(keys))


def test_aggregate_conserves_mass_and_boxes(oracle_mod):
    st = small_collision()
    import gcs
    pos, _ = gcs.pos_vel_from_stars(st)
    lo, hi = oracle_mod.bounds(pos)
    sk, idx = oracle_mod.sort(oracle_mod.encode(pos, lo, hi))
    sp = pos[idx]
    cl, cr, re, _, _ = oracle_mod.build(sk)
    for fp64 in (False, True):
        nodes, box = oracle_mod.aggregate(sp, cl, cr, re, com_fp64=fp64)
        np.testing.assert_allclose(nodes["mass"][0], sp[:, 3].astype(np.float64).sum(), rtol=1e-5)
        np.testing.assert_array_equal(box[0, :3], sp[:, :3].min(0))
        np.testing.assert_array_equal(box[0, 3:], sp[:, :3].max(0))
        com = (sp[:, :3].astype(np.float64) * sp[:, 3:4]).sum(0) / sp[:, 3].astype(np.float64).sum()
        np.testing.assert_allclose([nodes["com_x"][0], nodes["com_y"][0], nodes["com_z"][0]], com,
                                   atol=1e-4 if not fp64 else 1e-6)
        assert np.all(nodes["width"] >= 0)


def _tree_for(oracle_mod, pos):
    lo, hi = oracle_mod.bounds(pos)
    sk, idx = oracle_mod.sort(oracle_mod.encode(pos, lo, hi))
    sp = np.ascontiguousarray(pos[idx])
    cl, cr, re, _, _ = oracle_mod.build(sk)
    nodes, _ = oracle_mod.aggregate(sp, cl, cr, re)
    return sp, nodes


def test_walk_theta0_is_direct_sum(oracle_mod):
    """theta = 0 opens every node: the walk becomes the softened direct sum
    (with the reference's 1.01 eps^2 self exclusion)."""
    st = small_collision(256, 64, 32)
    import gcs
    pos, _ = gcs.pos_vel_from_stars(st)
    sp, nodes = _tree_for(oracle_mod, pos)
    eps2 = 0.01
    for L in (1, 8, 32):
        acc = oracle_mod.walk(sp, nodes, 1.0, eps2, 0.0, L)
        ex = oracle_mod.direct_fp64(sp, np.arange(len(sp)), 1.0, eps2)
        assert np.max(rel_err(acc[:, :3], ex)) < 2e-5


def test_walk_error_shrinks_with_theta(oracle_mod):
    st = small_collision()
    import gcs
    pos, _ = gcs.pos_vel_from_stars(st)
    sp, nodes = _tree_for(oracle_mod, pos)
    tg = np.arange(0, len(sp), 7)
    ex = oracle_mod.direct_fp64(sp, tg, 1.0, 0.0025)
    med = []
    for theta in (1.0, 0.7, 0.5, 0.3):
        acc = oracle_mod.walk(sp, nodes, 1.0, 0.0025, theta, 1)
        med.append(np.median(rel_err(acc[tg, :3], ex)))
    assert med[0] > med[1] > med[2] > med[3]
    assert med[2] < 1e-2


def test_integrate_and_colour_map(oracle_mod):
    n = 6
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    acc = np.zeros((n, 4), np.float32)
    speeds = [0.0, 60.0, 75.0, 140.0, 400.0, 10.0]
    types = [0, 0, 2, 2, 0, 1]
    vel[:, 0] = speeds
    tcol = np.array(types, np.uint32) | (np.uint32(7) << 8)
    vel[:, 3] = tcol.view(np.float32)
    x, v = oracle_mod.integrate(pos, vel, acc, 0.5)
    np.testing.assert_array_equal(x[:, 0], np.float32(0.5) * np.array(speeds, np.float32))
    t = v[:, 3].copy().view(np.uint32)
    rgb = [((c >> 8) & 255, (c >> 16) & 255, (c >> 24) & 255) for c in t]
    assert rgb[0] == (255, 50, 0)            # fire, t=0
    assert rgb[1] == (255, 170, 0)           # fire, t=0.4: g = 50 + 150*0.8
    assert rgb[2] == (0, 200, 255)           # ice, t=0.5 -> second branch, nt=0
    assert rgb[4] == (255, 255, 150)         # fire saturates at t=1
    assert rgb[5] == (7, 0, 0)               # dark matter keeps its colour


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ref_gpu_*.npz"))))
def test_oracle_matches_reference_gpu_golden(oracle_mod, path):
    """Stage outputs of the reference's own GPU engine on seeded inputs."""
    import gcs
    g = np.load(path)
    st = g["stars"]
    G, eps2, theta, dt, lo, hi = [float(x) for x in g["params"]]
    n = len(st)
    pos, vel = gcs.pos_vel_from_stars(st)
    keys = oracle_mod.encode(pos, lo, hi)
    sk, idx = oracle_mod.sort(keys)
    np.testing.assert_array_equal(sk, g["keys"])
    np.testing.assert_array_equal(idx.astype(np.int32), g["perm"])
    cl, cr, re, par, lp = oracle_mod.build(sk)
    ref_nodes = g["nodes"]
    np.testing.assert_array_equal(cl, ref_nodes["child_left"][: n - 1])
    np.testing.assert_array_equal(cr, ref_nodes["child_right"][: n - 1])
    ref_build = g["build"]
    np.testing.assert_array_equal(par[1:], ref_build["parent"][1 : n - 1])
    np.testing.assert_array_equal(lp, ref_build["parent"][n - 1 :])
    sp = np.ascontiguousarray(pos[idx])
    nodes, box = oracle_mod.aggregate(sp, cl, cr, re, com_fp64=False)
    np.testing.assert_array_equal(nodes["mass"], ref_nodes["mass"][: n - 1])
    np.testing.assert_array_equal(nodes["width"], ref_nodes["width"][: n - 1])
    np.testing.assert_array_equal(box[:, :3], ref_build["min"][: n - 1])
    np.testing.assert_array_equal(box[:, 3:], ref_build["max"][: n - 1])
    # the FP32 centre-of-mass formula rounds exactly as the reference's
    for a in ("com_x", "com_y", "com_z"):
        np.testing.assert_array_equal(nodes[a], ref_nodes[a][: n - 1], err_msg=a)
    # walk on the reference's own tree: same opening decisions, FP32 rounding only
    tree = ref_nodes[: n - 1].copy()
    tree["range_end"] = re
    acc = oracle_mod.walk(sp, tree, G, eps2, theta, 1)
    ra = g["accels"]
    scale = np.median(np.linalg.norm(ra, axis=1))
    err = rel_err(acc[:, :3], ra, floor=1e-3 * scale)
    assert np.percentile(err, 99.9) < 1e-5, np.percentile(err, 99.9)
    assert err.max() < 1e-4, err.max()
    # kick + drift + colour map is bit-exact given the reference's accelerations
    a4 = np.zeros((n, 4), np.float32)
    a4[:, :3] = ra
    x1, v1 = oracle_mod.integrate(sp, vel[idx], a4, dt, True)
    soa, rgbt = g["soa"], g["rgbt"]
    for k in range(3):
        np.testing.assert_array_equal(x1[:, k], soa[k])
        np.testing.assert_array_equal(v1[:, k], soa[3 + k])
    tcol = v1[:, 3].copy().view(np.uint32)
    for k in range(3):
        np.testing.assert_array_equal(((tcol >> (8 * (k + 1))) & 255).astype(np.uint8), rgbt[k])
    np.testing.assert_array_equal((tcol & 255).astype(np.uint8), rgbt[3])
