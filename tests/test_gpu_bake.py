"""Bake (gcs_bake): steps written as simulation.bin frames through the
pipelined path (device-side PlaybackStar packing, asynchronous copies into two
pinned buffers, a writer thread) are byte-identical to stepping and reading
each frame back one at a time (the reference's Bake loop, main.cpp:119-297)."""
import numpy as np
import pytest

from conftest import small_collision

pytestmark = pytest.mark.gpu


def _params(gcs):
    return gcs.reference_params(theta=0.5, epsilon_sq=0.05 ** 2, dt=0.005, leaf_size=4,
                                bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=1)


def _frames_one_at_a_time(gcs, stars, frames):
    p = _params(gcs)
    out = []
    with gcs.Context(len(stars)) as ctx:
        ctx.upload(stars)
        for _ in range(frames):
            ctx.step(p)
            out.append(ctx.download_playback())
    return np.concatenate(out).tobytes()


def test_bake_frames_equal_step_and_read(gcs_mod, tmp_path):
    gcs = gcs_mod
    stars = small_collision(2048, 512, 256, seed=31)
    want = _frames_one_at_a_time(gcs, stars, 5)
    path = tmp_path / "simulation.bin"
    with gcs.Context(len(stars)) as ctx:
        ctx.upload(stars)
        sec = ctx.bake(_params(gcs), 5, str(path))
        assert sec > 0.0
    data = path.read_bytes()
    assert len(data) == 5 * len(stars) * 16
    assert data == want
    frames = gcs.read_playback(str(path), len(stars))
    assert frames.shape[0] == 5


def test_bake_append_and_empty(gcs_mod, tmp_path):
    gcs = gcs_mod
    stars = small_collision(512, 128, 64, seed=32)
    want = _frames_one_at_a_time(gcs, stars, 4)
    path = tmp_path / "sim.bin"
    with gcs.Context(len(stars)) as ctx:
        ctx.upload(stars)
        ctx.bake(_params(gcs), 0, str(path))
        assert path.read_bytes() == b""
        ctx.bake(_params(gcs), 1, str(path), append=True)
        ctx.bake(_params(gcs), 3, str(path), append=True)
    assert path.read_bytes() == want


def test_bake_with_graphs_and_segments(gcs_mod, tmp_path):
    import torch
    gcs = gcs_mod
    a = small_collision(700, 170, 90, seed=33)
    b = small_collision(300, 60, 40, seed=34)
    s = torch.cuda.Stream()
    path = tmp_path / "two.bin"
    with gcs.Context(len(a) + len(b), max_segments=2) as ctx:
        ctx.set_stream(s.cuda_stream)
        ctx.set_graphs(True)
        ctx.set_segments([len(a), len(b)])
        ctx.upload(np.concatenate([a, b]))
        ctx.bake(_params(gcs), 3, str(path))
    frames = gcs.read_playback(str(path), len(a) + len(b))
    solo = np.frombuffer(_frames_one_at_a_time(gcs, b, 3), gcs.PLAYBACK_DTYPE).reshape(3, len(b))
    assert np.array_equal(frames[:, len(a):], solo)


def test_bake_rejects_bad_output(gcs_mod, tmp_path):
    gcs = gcs_mod
    stars = small_collision(256, 64, 32, seed=35)
    with gcs.Context(len(stars)) as ctx:
        ctx.upload(stars)
        with pytest.raises(gcs.GcsError):
            ctx.bake(_params(gcs), 1, str(tmp_path / "no_such_dir" / "x.bin"))
