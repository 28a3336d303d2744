"""Playback on the GPU: a baked simulation.bin read back with the reader
(gcs_playback_*) holds, frame by frame, the stepped state's positions,
colours and types; a frame copied to the device renders
(gcs_render_playback) exactly as the Stars it was written from
(gcs_render_stars), as the reference's Playback mode draws a frame's records
as those Stars (main.cpp:423-433)."""
import ctypes as C

import numpy as np
import pytest

from conftest import small_collision

pytestmark = pytest.mark.gpu


def test_baked_frames_read_back_and_render_as_their_stars(gcs_mod, tmp_path):
    import torch
    gcs = gcs_mod
    stars = small_collision(2048, 512, 256, seed=31)
    n = len(stars)
    p = gcs.reference_params(theta=0.5, epsilon_sq=0.05 ** 2, dt=0.005, leaf_size=4, walk_batch=64,
                             bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=1)
    path = tmp_path / "simulation.bin"
    stepped = []
    with gcs.Context(n) as ctx, gcs.Context(n) as solo:
        ctx.upload(stars)
        solo.upload(stars)
        ctx.bake(p, 3, str(path))
        for _ in range(3):
            solo.step(p)
            stepped.append(solo.download())
    with gcs.Playback(str(path), n) as pb:
        assert (pb.frames, pb.particles) == (3, n)
        frames = [pb.next() for _ in range(3)]
        assert pb.next().tobytes() == frames[0].tobytes()  # loops to the first frame

    cam = gcs.camera_reference()
    cam.pos[:] = (0.0, 30.0, 80.0)
    cam.front[:] = (0.0, -0.35, -1.0)
    w, h = 320, 200
    L = gcs.lib()
    for frame, st in zip(frames, stepped):
        for k in ("x", "y", "z", "r", "g", "b"):
            np.testing.assert_array_equal(frame[k], st[k], err_msg=k)
        np.testing.assert_array_equal(frame["padding"], st["type"])
        outs = []
        for fn, recs in ((L.gcs_render_playback, frame), (L.gcs_render_stars, st)):
            dev = torch.from_numpy(recs.view(np.uint8).copy()).cuda()
            acc = torch.zeros(h * w * 3, dtype=torch.int64, device="cuda")
            rgba = torch.zeros(h * w * 4, dtype=torch.uint8, device="cuda")
            rc = fn(C.c_void_p(dev.data_ptr()), n, C.byref(cam), w, h, C.c_void_p(acc.data_ptr()),
                    C.c_void_p(rgba.data_ptr()), None)
            assert rc == gcs.OK
            torch.cuda.synchronize()
            outs.append((acc.cpu().numpy(), rgba.cpu().numpy()))
        (acc_pb, img_pb), (acc_st, img_st) = outs
        assert np.array_equal(acc_pb, acc_st) and np.array_equal(img_pb, img_st)
        assert (acc_pb > 0).sum() > 1000  # a non-trivial frame

    # the reference's camera target for the frame: FP64 mean position as float
    want = []
    for axis in ("x", "y", "z"):
        s = 0.0
        for v in stepped[-1][axis]:
            s += float(v)
        want.append(np.float32(s / n))
    np.testing.assert_array_equal(gcs.playback_centre(frames[-1]), np.array(want, np.float32))

