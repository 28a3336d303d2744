"""The simulation.bin reader (gcs_playback_*), host only: frame counts from
the file size (and the reference's inference from a frame count), and the
reference Playback mode's navigation (main.cpp:397-419) against a model of
its file-offset arithmetic: forward reads loop to the first frame after the
last, a backward step moves the offset back two frames or to the last
frame.  The camera target is the reference's FP64 mean (main.cpp:435-441)."""
import ctypes as C

import numpy as np
import pytest


def _frames(gcs, n, count, seed=0):
    rng = np.random.default_rng(seed)
    f = np.zeros((count, n), dtype=gcs.PLAYBACK_DTYPE)
    for k in range(count):
        f["x"][k] = k  # the frame index, to see which frame came back
        f["y"][k] = rng.normal(size=n)
        f["z"][k] = rng.normal(size=n)
        f["r"][k], f["g"][k], f["b"][k] = rng.integers(0, 256, (3, n))
        f["padding"][k] = rng.integers(0, 3, n)
    return f


class _ReferenceModel:
    """main.cpp's playback offsets, in bytes."""

    def __init__(self, data: bytes, n: int):
        self.d, self.fs, self.off = data, 16 * n, 0

    def forward(self):
        if self.off + self.fs > len(self.d):  # fread came back short: loop to the start
            self.off = 0
        out = self.d[self.off:self.off + self.fs]
        self.off += self.fs
        return out

    def backward(self):
        new = self.off - 2 * self.fs
        if new < 0:
            new = len(self.d) - self.fs
        self.off = new
        return self.forward()


def test_navigation_matches_reference_offsets(gcs_mod, tmp_path):
    gcs = gcs_mod
    n, count = 37, 7
    f = _frames(gcs, n, count)
    path = tmp_path / "simulation.bin"
    f.tofile(path)
    model = _ReferenceModel(path.read_bytes(), n)
    rng = np.random.default_rng(1)
    with gcs.Playback(str(path), n) as pb:
        assert (pb.frames, pb.particles, pb.position) == (count, n, 0)
        first_back = pb.prev()  # backward before any read: the last frame
        assert first_back.tobytes() == model.backward()
        assert first_back["x"][0] == count - 1 and pb.position == 0
        for _ in range(300):
            if rng.random() < 0.65:
                got, want = pb.next(), model.forward()
            else:
                got, want = pb.prev(), model.backward()
            assert got.tobytes() == want
            assert pb.position == (model.off // model.fs) % count


def test_forward_loops_and_seek(gcs_mod, tmp_path):
    gcs = gcs_mod
    n, count = 5, 4
    f = _frames(gcs, n, count, seed=2)
    path = tmp_path / "s.bin"
    f.tofile(path)
    with gcs.Playback(str(path), n) as pb:
        seen = [int(pb.next()["x"][0]) for _ in range(2 * count + 1)]
        assert seen == [k % count for k in range(2 * count + 1)]
        for target in (2, -1, count + 3, 0):
            pb.seek(target)
            assert pb.position == target % count
            got = pb.next()
            assert got.tobytes() == f[target % count].tobytes()
        np.testing.assert_array_equal(gcs.read_playback(str(path), n), f)


def test_frame_count_inference(gcs_mod, tmp_path):
    """particles = 0: the reference's n = size / frames / 16 (main.cpp:309)."""
    gcs = gcs_mod
    n = 3
    f = _frames(gcs, n, 2000, seed=3)
    path = tmp_path / "baked.bin"
    f.tofile(path)
    with gcs.Playback(str(path), 0, 2000) as pb:
        assert (pb.particles, pb.frames) == (n, 2000)
        assert pb.next().tobytes() == f[0].tobytes()
    with open(path, "ab") as fh:  # a trailing partial record: whole frames are kept
        fh.write(bytes(5))
    with gcs.Playback(str(path), 0, 2000) as pb:
        assert (pb.particles, pb.frames) == (n, 2000)
        pb.seek(-1)
        assert pb.next().tobytes() == f[-1].tobytes()


def test_bad_files_and_arguments(gcs_mod, tmp_path):
    gcs = gcs_mod
    f = _frames(gcs, 4, 3, seed=4)
    path = tmp_path / "s.bin"
    f.tofile(path)
    with pytest.raises(gcs.GcsError):
        gcs.Playback(str(path), 5)  # 3 x 4 records are not whole frames of 5
    with pytest.raises(gcs.GcsError):
        gcs.Playback(str(tmp_path / "missing.bin"), 4)
    empty = tmp_path / "empty.bin"
    empty.write_bytes(b"")
    with pytest.raises(gcs.GcsError):
        gcs.Playback(str(empty), 4)
    with pytest.raises(gcs.GcsError):
        gcs.Playback(str(path), -1)
    with pytest.raises(gcs.GcsError):
        gcs.Playback(str(path), 0, 0)
    with pytest.raises(gcs.GcsError):
        gcs.Playback(str(path), 0, 10 ** 6)  # inference leaves fewer than one record per frame


def test_camera_target_is_the_reference_mean(gcs_mod):
    gcs = gcs_mod
    f = _frames(gcs, 1001, 1, seed=5)[0]
    f["x"] = np.random.default_rng(6).normal(50.0, 20.0, len(f))
    want = []
    for axis in ("x", "y", "z"):
        s = 0.0
        for v in f[axis]:
            s += float(v)  # the reference's serial double sum
        want.append(np.float32(s / len(f)))
    np.testing.assert_array_equal(gcs.playback_centre(f), np.array(want, np.float32))


def test_render_playback_rejects_bad_arguments(gcs_mod):
    """Argument checks come before any device work (no GPU needed)."""
    gcs = gcs_mod
    L = gcs.lib()
    cam = gcs.camera_reference()
    acc = np.zeros(8 * 8 * 3, np.uint64)
    assert L.gcs_render_playback(None, 10, C.byref(cam), 8, 8, acc.ctypes.data, None, None) != gcs.OK
    assert L.gcs_render_playback(acc.ctypes.data, 1, C.byref(cam), 0, 8, acc.ctypes.data, None, None) != gcs.OK
    assert L.gcs_render_playback(acc.ctypes.data + 4, 1, C.byref(cam), 8, 8, acc.ctypes.data, None, None) != gcs.OK


def test_camera_locks_on_the_frame_centre(gcs_mod):
    """renderer.cpp:255-256: front = normalize(target - pos); the view then
    puts the target on the axis in front of the eye."""
    gcs = gcs_mod
    cam = gcs.camera_reference()
    target = np.array([12.5, -3.0, 40.0], np.float32)
    gcs.camera_look_at(cam, target)
    d = target - np.array(cam.pos[:], np.float32)
    want = d * (np.float32(1.0) / np.sqrt(np.float32(d @ d), dtype=np.float32))
    np.testing.assert_allclose(np.array(cam.front[:], np.float32), want, rtol=2e-7, atol=0)
    v, _ = gcs.camera_matrices(cam, 640, 360)
    eye = v @ np.append(target, np.float32(1.0)).astype(np.float64)
    assert abs(eye[0]) < 1e-3 and abs(eye[1]) < 1e-3 and eye[2] < 0
    with pytest.raises(gcs.GcsError):
        gcs.camera_look_at(cam, cam.pos[:])
