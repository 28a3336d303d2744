"""The host step with the Star transfer overlapped with the walk (gcs_step_host).

The walk's epilogue applies the kick/drift out of place and writes the Star
records: straight into the caller's array when it is pinned, device-mapped
host memory (16-byte aligned), else into device staging, from which the host
copies each finished chunk of walk groups while the walk runs.  The Stars it returns, and the state it leaves on the device, must be
the same bits as the plain stage sequence (bounds .. integrate) followed by
gcs_download_stars, step after step: for one and several segments, both
group widths, ragged sizes (1, 2, 33 particles; groups that do not fill a
chunk), with graph-captured steps in between, and through the reference's
own entry point (cuda_physics_step)."""
import ctypes as C

import numpy as np
import pytest

from conftest import small_collision

pytestmark = pytest.mark.gpu


def _params(gcs, leaf=4, batch=64):
    return gcs.reference_params(theta=0.5, epsilon_sq=0.05 ** 2, dt=0.005, leaf_size=leaf, walk_batch=batch,
                                bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=1)


def _pinned_stars(gcs, n, byte_offset=0):
    """A Star array in pinned host memory (optionally starting byte_offset
    bytes into the pinned block)."""
    import torch
    block = torch.zeros(n * 32 + 64, dtype=torch.uint8, pin_memory=True)
    arr = block.numpy()[byte_offset:byte_offset + n * 32].view(gcs.STAR_DTYPE)
    return block, arr


def _pair(gcs, stars, counts, width, p, steps, graphs_every=0, pinned=False, byte_offset=0):
    n = len(stars)
    with gcs.Context(n, max_segments=len(counts)) as a, gcs.Context(n, max_segments=len(counts)) as b:
        for ctx in (a, b):
            ctx.set_segments(counts)
            ctx.set_group_width(width)
            ctx.upload(stars)
        if pinned:
            keep, out = _pinned_stars(gcs, n, byte_offset)
        else:
            out = np.zeros(n, dtype=gcs.STAR_DTYPE)
        for k in range(steps):
            if graphs_every and k % graphs_every == graphs_every - 1:
                # a plain (graph-captured) step on the overlapped context
                # keeps the two in step through the ping-pong arrays
                import torch
                s = torch.cuda.Stream()
                a.set_stream(s.cuda_stream)
                a.set_graphs(True)
                a.step(p)
                a.synchronize()
                a.set_graphs(False)
                a.set_stream(0)
                b.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_INTEGRATE)
                continue
            out[:] = 0
            a.step_host(p, out)
            b.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_INTEGRATE)
            ref = b.download()
            assert out.tobytes() == ref.tobytes(), "step %d: Stars differ" % k
            assert a.download().tobytes() == ref.tobytes(), "step %d: device state differs" % k
            assert a.device_status() == 0
        assert a.download().tobytes() == b.download().tobytes()


@pytest.mark.parametrize("width", [32, 64])
@pytest.mark.parametrize("pinned", [False, True])
def test_overlapped_host_step_equals_plain_step(gcs_mod, width, pinned):
    gcs = gcs_mod
    stars = small_collision(3000, 700, 300, seed=17)  # 8,000 particles, 250 or 125 groups
    _pair(gcs, stars, [len(stars)], width, _params(gcs), steps=4, pinned=pinned)


@pytest.mark.parametrize("byte_offset", [32, 8])
def test_pinned_array_inside_a_block(gcs_mod, byte_offset):
    """A pinned array one Star into its block is written directly; one that
    starts 8 bytes in (not 16-byte aligned) takes the copy path; both give
    the same bytes."""
    gcs = gcs_mod
    stars = small_collision(3000, 700, 300, seed=25)
    _pair(gcs, stars, [len(stars)], 32, _params(gcs), steps=2, pinned=True, byte_offset=byte_offset)


@pytest.mark.parametrize("width,leaf,theta,pot", [(16, 1, 0.5, 0), (48, 32, 0.7, 0), (32, 4, 0.0, 0),
                                                   (64, 8, 0.5, 1)])
@pytest.mark.parametrize("pinned", [False, True])
def test_overlapped_host_step_settings(gcs_mod, width, leaf, theta, pot, pinned):
    """Other group widths (two targets a lane above 32), leaf sizes, theta 0
    (every node opened) and potentials: the same bits as the plain step."""
    gcs = gcs_mod
    stars = small_collision(1500, 350, 150, seed=26)  # 4,000 particles
    p = gcs.reference_params(theta=theta, epsilon_sq=0.05 ** 2, dt=0.005, leaf_size=leaf, walk_batch=64,
                             bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=1, with_potential=pot)
    _pair(gcs, stars, [len(stars)], width, p, steps=2, pinned=pinned)


def test_overlapped_host_step_many_chunks(gcs_mod):
    gcs = gcs_mod
    stars = small_collision(30000, 7000, 3000, seed=18)  # 80,000 particles: 2,500 groups, 48 chunks
    _pair(gcs, stars, [len(stars)], 32, _params(gcs), steps=2)


def test_overlapped_host_step_head_and_tail_chunks(gcs_mod):
    """400,000 particles: 12,500 groups, more than twice the walk's resident
    warps, so both the large head chunks and the small tail chunks are used."""
    gcs = gcs_mod
    stars = small_collision(150000, 37500, 12500, seed=24)
    _pair(gcs, stars, [len(stars)], 32, _params(gcs), steps=2)


def test_overlapped_host_step_segments(gcs_mod):
    gcs = gcs_mod
    stars = small_collision(3000, 700, 300, seed=19)
    counts = [5000, 33, 1, 2966]
    _pair(gcs, stars, counts, 32, _params(gcs, leaf=8, batch=32), steps=3)
    _pair(gcs, stars, counts, 32, _params(gcs, leaf=8, batch=32), steps=3, pinned=True)


@pytest.mark.parametrize("n", [1, 2, 33, 1000])
@pytest.mark.parametrize("pinned", [False, True])
def test_overlapped_host_step_ragged(gcs_mod, n, pinned):
    gcs = gcs_mod
    stars = small_collision(3000, 700, 300, seed=20)[:n].copy()
    _pair(gcs, stars, [n], 32, _params(gcs), steps=2, pinned=pinned)


def test_overlapped_host_step_between_graph_steps(gcs_mod):
    gcs = gcs_mod
    stars = small_collision(3000, 700, 300, seed=21)
    _pair(gcs, stars, [len(stars)], 32, _params(gcs), steps=6, graphs_every=2)


def test_host_step_over_a_step_range(gcs_mod):
    """A slice of the scenario (gcs_set_step_range) takes the plain sequence."""
    gcs = gcs_mod
    stars = small_collision(3000, 700, 300, seed=22)
    n = len(stars)
    p = _params(gcs)
    with gcs.Context(n) as a, gcs.Context(n) as b:
        for ctx in (a, b):
            ctx.upload(stars)
            ctx.set_step_range(0, 4096)
        out = np.zeros(n, dtype=gcs.STAR_DTYPE)
        for _ in range(2):
            a.step_host(p, out)
            b.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_INTEGRATE)
            assert out.tobytes() == b.download().tobytes()


def test_dropin_host_step_equals_engine_steps(gcs_mod):
    """cuda_physics_step (host Stars) against the engine's plain sequence with
    the drop-in's parameters."""
    gcs = gcs_mod
    L = gcs.lib()
    init = L._Z9cuda_initi
    init.restype, init.argtypes = C.c_bool, [C.c_int]
    cleanup = L._Z12cuda_cleanupv
    cleanup.restype, cleanup.argtypes = None, []
    upload = L._Z25cuda_upload_initial_starsPK4Stari
    upload.restype, upload.argtypes = None, [C.c_void_p, C.c_int]
    step = L._Z17cuda_physics_stepP4Starifffffb
    step.restype = C.c_float
    step.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_bool]
    stars = small_collision(3000, 700, 300, seed=23)
    n = len(stars)
    pos, _ = gcs.pos_vel_from_stars(stars)
    lo, hi = float(pos[:, :3].min()), float(pos[:, :3].max())
    assert init(n)
    try:
        upload(stars.ctypes.data, n)
        keep, host = _pinned_stars(gcs, n)  # the Bake driver's pinned array
        p = gcs.Params()
        L.gcs_params_reference(C.byref(p))
        p.G, p.epsilon_sq, p.dt, p.global_min, p.global_max = 1.0, 10.0, 0.01, lo, hi
        with gcs.Context(n) as b:
            b.upload(stars)
            for _ in range(3):
                step(host.ctypes.data, n, 1.0, 10.0, 0.01, lo, hi, False)
                b.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_INTEGRATE)
                assert host.tobytes() == b.download().tobytes()
    finally:
        cleanup()


@pytest.mark.parametrize("pinned,same_buffer,bounds", [(True, True, "device"), (False, True, "device"),
                                                        (True, False, "caller"), (False, False, "device")])
def test_host_step_io_equals_upload_then_host_step(gcs_mod, pinned, same_buffer, bounds):
    """gcs_step_host_io (chunked upload, each chunk unpacked and reduced into
    the bounds as it lands, then the host step) gives the same Stars and the
    same device state as gcs_upload_stars + gcs_step_host, step after step,
    over uneven segments (chunks of the upload cross segment ends)."""
    gcs = gcs_mod
    parts = [small_collision(9000, 2000, 1000, seed=61), small_collision(700, 150, 60, seed=62)[:1777],
             small_collision(20, 5, 3, seed=63)[:33]]
    stars = np.concatenate(parts)
    counts = [len(x) for x in parts]
    n = len(stars)
    p = _params(gcs)
    if bounds == "caller":
        pos, _ = gcs.pos_vel_from_stars(stars)
        p.bounds_mode = gcs.BOUNDS_CALLER
        p.global_min, p.global_max = float(pos[:, :3].min()) - 1.0, float(pos[:, :3].max()) + 1.0
        counts = [n]
    with gcs.Context(n, max_segments=len(counts)) as a, gcs.Context(n, max_segments=len(counts)) as b:
        for ctx in (a, b):
            ctx.set_segments(counts)
        if pinned:
            keep_in, cur = _pinned_stars(gcs, n)
            keep_out, out = _pinned_stars(gcs, n, 16)
        else:
            cur, out = np.zeros(n, dtype=gcs.STAR_DTYPE), np.zeros(n, dtype=gcs.STAR_DTYPE)
        cur[:] = stars
        ref = stars.copy()
        ref_out = np.zeros(n, dtype=gcs.STAR_DTYPE)
        for _ in range(3):
            dst = cur if same_buffer else out
            a.step_host_io(p, cur, dst)
            b.upload(ref)
            b.step_host(p, ref_out)
            assert dst.tobytes() == ref_out.tobytes()
            assert a.download().tobytes() == b.download().tobytes()
            cur[:] = dst
            ref[:] = ref_out
        assert a.device_status() == 0 and b.device_status() == 0
