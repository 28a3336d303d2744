"""Headless splat renderer, CPU side: the camera matrices of the C ABI and the
oracle's restatement of the reference's GL point pipeline (renderer.cpp:97-148,
203, 248, 262-263) against an independent float64 evaluation of the same
formulas on hand-placed stars."""
import math

import numpy as np
import pytest

UNIT = 2.0 ** 24


def _lookat(eye, front, up):
    f = np.asarray(front, np.float64)
    f = f / np.linalg.norm(f)
    s = np.cross(f, up)
    s = s / np.linalg.norm(s)
    u = np.cross(s, f)
    e = np.asarray(eye, np.float64)
    return np.array([[*s, -s @ e], [*u, -u @ e], [*(-f), f @ e], [0, 0, 0, 1]])


def _perspective(fovy_deg, aspect, n, f):
    t = math.tan(math.radians(fovy_deg) / 2)
    return np.array([[1 / (aspect * t), 0, 0, 0], [0, 1 / t, 0, 0],
                     [0, 0, -(f + n) / (f - n), -2 * f * n / (f - n)], [0, 0, -1, 0]])


def _star(gcs, x, y, z, typ=0, rgb=(255, 128, 0)):
    s = np.zeros(1, gcs.STAR_DTYPE)
    s["x"], s["y"], s["z"] = x, y, z
    s["mass"] = 1.0
    s["type"] = typ
    s["r"], s["g"], s["b"] = rgb
    return s


def test_camera_matrices_are_lookat_and_perspective(gcs_mod):
    gcs = gcs_mod
    cam = gcs.camera_reference()
    assert tuple(cam.pos) == (0.0, 150.0, 600.0) and cam.fovy_deg == 45.0
    v, p = gcs.camera_matrices(cam, 1920, 1080)
    vr = _lookat(cam.pos, cam.front, cam.up)
    pr = _perspective(45.0, 1920 / 1080, 0.1, 5000.0)
    np.testing.assert_allclose(v, vr, rtol=1e-6, atol=1e-4)
    np.testing.assert_allclose(p, pr, rtol=1e-6, atol=1e-7)
    # the eye maps to the view-space origin; near and far planes to ndc z = -1, +1
    np.testing.assert_allclose(vr @ [*cam.pos, 1.0], [0, 0, 0, 1], atol=1e-9)
    for z, want in ((-0.1, -1.0), (-5000.0, 1.0)):
        c = pr @ [0.0, 0.0, z, 1.0]
        assert abs(c[2] / c[3] - want) < 1e-9


def test_camera_rejects_degenerate_input(gcs_mod):
    gcs = gcs_mod
    cam = gcs.camera_reference()
    cam.up[:] = (0.0, -0.2, -1.0)  # parallel to the view direction
    with pytest.raises(gcs.GcsError):
        gcs.camera_matrices(cam, 64, 64)
    cam = gcs.camera_reference()
    cam.z_far = cam.z_near
    with pytest.raises(gcs.GcsError):
        gcs.camera_matrices(cam, 64, 64)


def _expected_fragments(star_xyz, typ, rgb, v, p, w, h):
    """Float64 evaluation of one star's fragments: {(i, j): (r, g, b) contributions}."""
    vs = v @ [*star_xyz, 1.0]
    d = np.linalg.norm(vs[:3])
    size = min(max(2500.0 / d, 1.0), 6.0) if typ == 1 else min(max(1000.0 / d, 1.0), 3.0)
    c = p @ vs
    if not (c[3] > 0 and all(abs(c[k]) <= c[3] for k in range(3))):
        return {}
    xw = (c[0] / c[3] + 1) * 0.5 * w
    yw = (c[1] / c[3] + 1) * 0.5 * h
    col = np.array([0.4, 0.0, 0.8]) if typ == 1 else np.asarray(rgb) / 255.0
    amul = 0.03 if typ == 1 else 0.15
    out = {}
    for j in range(h):
        for i in range(w):
            cx, cy = i + 0.5, j + 0.5
            if not (xw - size / 2 <= cx < xw + size / 2 and yw - size / 2 <= cy < yw + size / 2):
                continue
            r2 = (2 * (cx - xw) / size) ** 2 + (2 * (cy - yw) / size) ** 2
            if r2 > 1.0:
                continue
            out[(i, j)] = col * math.exp(-3 * r2) * amul
    return out


@pytest.mark.parametrize("typ,dist", [(0, 500.0), (0, 200.0), (1, 300.0), (1, 1200.0), (2, 600.0)])
def test_oracle_splat_of_one_star(gcs_mod, oracle_mod, typ, dist):
    gcs = gcs_mod
    cam = gcs.camera_reference()
    w, h = 48, 40
    v, p = gcs.camera_matrices(cam, w, h)
    f = np.asarray(cam.front, np.float64)
    pos = np.asarray(cam.pos, np.float64) + dist * f / np.linalg.norm(f) + [0.37, -0.21, 0.0]
    s = _star(gcs, *pos, typ=typ, rgb=(250, 120, 30))
    acc, rgba = oracle_mod.render(s, v, p, w, h)
    exp = _expected_fragments(pos, typ, (250, 120, 30), v.astype(np.float64), p.astype(np.float64), w, h)
    assert exp, "the star must be on screen"
    lit = {(i, j) for j, i in zip(*np.nonzero(acc.sum(axis=2)))}
    assert lit == {k for k, val in exp.items() if np.any(np.rint(val * UNIT) > 0)}
    for (i, j), val in exp.items():
        np.testing.assert_allclose(acc[j, i].astype(np.float64), val * UNIT, rtol=1e-5, atol=2.0)
    clear = np.rint(np.array([0.01, 0.01, 0.02], np.float32).astype(np.float64) * 255)
    untouched = acc.sum(axis=2) == 0
    assert np.all(rgba[untouched][:, :3] == clear) and np.all(rgba[..., 3] == 255)


def test_oracle_culls_points_outside_the_clip_volume(gcs_mod, oracle_mod):
    gcs = gcs_mod
    cam = gcs.camera_reference()
    w, h = 32, 32
    v, p = gcs.camera_matrices(cam, w, h)
    eye = np.asarray(cam.pos, np.float64)
    f = np.asarray(cam.front, np.float64) / np.linalg.norm(cam.front)
    stars = np.concatenate([
        _star(gcs, *(eye - 50.0 * f)),              # behind the eye
        _star(gcs, *(eye + 6000.0 * f)),            # beyond the far plane
        _star(gcs, *(eye + 0.05 * f)),              # in front of the near plane
        _star(gcs, *(eye + 100.0 * f + [500.0, 0.0, 0.0])),  # far outside the field of view
        _star(gcs, float("nan"), 0.0, 0.0),         # not a position
    ])
    acc, _ = oracle_mod.render(stars, v, p, w, h)
    assert acc.sum() == 0


def test_oracle_drops_fragments_outside_the_viewport(gcs_mod, oracle_mod):
    gcs = gcs_mod
    cam = gcs.camera_reference()
    w, h = 40, 30
    v, p = gcs.camera_matrices(cam, w, h)
    # a dark-matter point (6 px) whose centre sits just inside the left edge
    vs_target = np.array([0.0, 0.0, -300.0, 1.0])
    c = p.astype(np.float64) @ vs_target
    x_ndc = -1.0 + 1.0 / w  # half a pixel in from the left edge
    vs_target[0] = x_ndc * c[3] / p[0, 0]
    world = np.linalg.solve(v.astype(np.float64), vs_target)[:3]
    s = _star(gcs, *world, typ=1)
    acc, _ = oracle_mod.render(s, v, p, w, h)
    exp = _expected_fragments(world, 1, (0, 0, 0), v.astype(np.float64), p.astype(np.float64), w, h)
    lit = {(i, j) for j, i in zip(*np.nonzero(acc.sum(axis=2)))}
    assert lit and all(i < 4 for i, _ in lit)
    assert lit == {k for k, val in exp.items() if np.any(np.rint(val * UNIT) > 0)}


def test_oracle_frame_is_order_independent(gcs_mod, oracle_mod):
    gcs = gcs_mod
    stars = gcs.collision_equal(512, 128, 64, seed=3)
    cam = gcs.camera_reference()
    cam.pos[:] = (0.0, 30.0, 80.0)
    cam.front[:] = (0.0, -0.35, -1.0)
    v, p = gcs.camera_matrices(cam, 96, 64)
    a1, r1 = oracle_mod.render(stars, v, p, 96, 64)
    perm = np.random.default_rng(0).permutation(len(stars))
    a2, r2 = oracle_mod.render(stars[perm], v, p, 96, 64)
    assert np.array_equal(a1, a2) and np.array_equal(r1, r2)
    assert (a1.sum(axis=2) > 0).sum() > 500


def test_write_ppm_round_trip(gcs_mod, tmp_path):
    gcs = gcs_mod
    rgba = np.random.default_rng(1).integers(0, 256, (5, 7, 4), dtype=np.uint8)
    path = tmp_path / "f.ppm"
    gcs.write_ppm(str(path), rgba)
    data = path.read_bytes()
    head, body = data[:len(b"P6\n7 5\n255\n")], data[len(b"P6\n7 5\n255\n"):]
    assert head == b"P6\n7 5\n255\n"
    img = np.frombuffer(body, np.uint8).reshape(5, 7, 3)
    assert np.array_equal(img, rgba[::-1, :, :3])
