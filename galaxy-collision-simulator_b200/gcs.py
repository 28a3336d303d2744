"""ctypes binding of libgcs.so (include/gcs.h) - the Python mirror of the
engine's C ABI, used by the tests and bench.py.

The engine is native code; this module only marshals arguments.  It raises
if the library is missing or a call fails - there is no Python fallback.
The record dtypes mirror include/gcs_types.h byte for byte.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgcs.so")

STAR_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("vx", "<f4"), ("vy", "<f4"),
                       ("vz", "<f4"), ("mass", "<f4"), ("type", "u1"), ("r", "u1"), ("g", "u1"),
                       ("b", "u1")])
PLAYBACK_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("r", "u1"), ("g", "u1"),
                           ("b", "u1"), ("padding", "u1")])
NODE_DTYPE = np.dtype([("com_x", "<f4"), ("com_y", "<f4"), ("com_z", "<f4"), ("mass", "<f4"),
                       ("width", "<f4"), ("child_left", "<i4"), ("child_right", "<i4"),
                       ("range_end", "<i4")])
BUILD_DTYPE = np.dtype([("min_x", "<f4"), ("min_y", "<f4"), ("min_z", "<f4"), ("max_x", "<f4"),
                        ("max_y", "<f4"), ("max_z", "<f4"), ("flag", "<i4"), ("parent", "<i4")])
assert STAR_DTYPE.itemsize == 32 and PLAYBACK_DTYPE.itemsize == 16
assert NODE_DTYPE.itemsize == 32 and BUILD_DTYPE.itemsize == 32

OK = 0
BOUNDS_CALLER, BOUNDS_DEVICE = 0, 1
(STAGE_BOUNDS, STAGE_ENCODE, STAGE_SORT, STAGE_GATHER, STAGE_BUILD, STAGE_AGGREGATE, STAGE_WALK,
 STAGE_INTEGRATE) = range(8)
(BUF_KEYS, BUF_INDEX, BUF_NODES, BUF_BUILD, BUF_LEAF_PARENT, BUF_ACCEL, BUF_POS, BUF_VEL, BUF_BOUNDS,
 BUF_KEYS_UNSORTED) = range(10)
DEV_SORT_LOOKBACK_TIMEOUT, DEV_WALK_STACK_OVERFLOW, DEV_NONFINITE_POSITION, DEV_BUILD_RANGE = 1, 2, 4, 8
DEV_TREE_MALFORMED = 16


class Params(C.Structure):
    _fields_ = [("G", C.c_float), ("epsilon_sq", C.c_float), ("theta", C.c_float), ("dt", C.c_float),
                ("leaf_size", C.c_int32), ("bounds_mode", C.c_int32), ("global_min", C.c_float),
                ("global_max", C.c_float), ("recolor", C.c_int32), ("com_fp64", C.c_int32),
                ("walk_batch", C.c_int32), ("walk_blocks_per_sm", C.c_int32),
                ("with_potential", C.c_int32), ("tune_leaf_min", C.c_int32), ("reserved", C.c_int32 * 2)]


class GalaxySpec(C.Structure):
    _fields_ = [("n_disc", C.c_int64), ("n_bulge", C.c_int64), ("n_halo", C.c_int64),
                ("disc_mass", C.c_float), ("disc_a", C.c_float), ("disc_b", C.c_float),
                ("disc_rmax", C.c_float), ("disc_zmax", C.c_float), ("bulge_mass", C.c_float),
                ("bulge_a", C.c_float), ("bulge_rmax", C.c_float), ("halo_mass", C.c_float),
                ("halo_a", C.c_float), ("halo_rmax", C.c_float), ("pos", C.c_float * 3),
                ("vel", C.c_float * 3), ("incline_deg", C.c_float), ("type", C.c_uint8)]


class CollisionSpec(C.Structure):
    _fields_ = [("galaxy", GalaxySpec * 2), ("seed", C.c_uint64), ("G", C.c_float),
                ("disc_dispersion", C.c_float)]


class Camera(C.Structure):
    """gcs_camera: eye, view direction (looks at pos + front), up, vertical
    field of view in degrees, near and far planes (renderer.cpp:9-11, 262-263)."""
    _fields_ = [("pos", C.c_float * 3), ("front", C.c_float * 3), ("up", C.c_float * 3),
                ("fovy_deg", C.c_float), ("z_near", C.c_float), ("z_far", C.c_float)]


class ServerResult(C.Structure):
    _fields_ = [("id", C.c_uint64), ("n", C.c_int64), ("steps", C.c_int32), ("status", C.c_int32),
                ("queued_ms", C.c_double), ("latency_ms", C.c_double)]


class GcsError(RuntimeError):
    pass


_lib = None


def lib() -> C.CDLL:
    """Load libgcs.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GcsError("libgcs.so not built: run __graft_entry__.build() or make -C %s" % HERE)
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    i32, i64, u64, f32 = C.c_int32, C.c_int64, C.c_uint64, C.c_float
    sig = {
        "gcs_params_reference": (None, [C.POINTER(Params)]),
        "gcs_create": (C.c_int, [C.POINTER(P), i64, i32, i32]),
        "gcs_destroy": (None, [P]),
        "gcs_set_stream": (C.c_int, [P, P]),
        "gcs_get_stream": (P, [P]),
        "gcs_status_string": (C.c_char_p, [C.c_int]),
        "gcs_last_error": (C.c_char_p, [P]),
        "gcs_set_segments": (C.c_int, [P, i32, C.POINTER(i64)]),
        "gcs_num_particles": (i64, [P]),
        "gcs_num_segments": (i32, [P]),
        "gcs_num_internal_nodes": (i64, [P]),
        "gcs_upload_stars": (C.c_int, [P, P, i64, i64]),
        "gcs_download_stars": (C.c_int, [P, P, i64, i64]),
        "gcs_download_playback": (C.c_int, [P, P, i64, i64]),
        "gcs_step": (C.c_int, [P, C.POINTER(Params)]),
        "gcs_step_host": (C.c_int, [P, C.POINTER(Params), P]),
        "gcs_step_host_io": (C.c_int, [P, C.POINTER(Params), P, P]),
        "gcs_compute_accels": (C.c_int, [P, C.POINTER(Params)]),
        "gcs_kick": (C.c_int, [P, f32]),
        "gcs_run_stages": (C.c_int, [P, C.POINTER(Params), i32, i32]),
        "gcs_synchronize": (C.c_int, [P]),
        "gcs_device_status": (C.c_int, [P, C.POINTER(C.c_uint32), i32]),
        "gcs_read_buffer": (C.c_int, [P, i32, P, i64, i64]),
        "gcs_collision_spec_equal": (C.c_int, [C.POINTER(CollisionSpec), i64, i64, i64, u64]),
        "gcs_collision_spec_pair": (C.c_int, [C.POINTER(CollisionSpec), i64, f32, f32, f32, f32, u64]),
        "gcs_collision_count": (i64, [C.POINTER(CollisionSpec)]),
        "gcs_generate_collision": (C.c_int, [C.POINTER(CollisionSpec), P, i64]),
        "gcs_diagnostics": (C.c_int, [P, i32, C.POINTER(C.c_double)]),
        "gcs_diagnostics_kicked": (C.c_int, [P, i32, C.c_double, C.POINTER(C.c_double)]),
        "gcs_direct_accels_fp64": (C.c_int, [P, C.POINTER(Params), i32, C.POINTER(i64), i64,
                                             C.POINTER(C.c_double)]),
        "gcs_count_interactions": (C.c_int, [P, C.POINTER(Params), C.POINTER(C.c_uint64)]),
        "gcs_walk_stack_peak": (C.c_int, [P, C.POINTER(C.c_int64)]),
        "gcs_walk_lane_use": (C.c_int, [P, C.POINTER(C.c_uint64)]),
        "gcs_autotune": (C.c_int, [P, C.POINTER(Params), C.POINTER(C.c_double)]),
        "gcs_set_group_width": (C.c_int, [P, i32]),
        "gcs_set_walk_frontier": (C.c_int, [P, i32]),
        "gcs_group_width": (i32, [P]),
        "gcs_sort_pairs_static": (C.c_int, [P, P, P, P, i64, P, P]),
        "gcs_set_graphs": (C.c_int, [P, i32]),
        "gcs_set_walk_events": (C.c_int, [P, C.c_void_p, C.c_void_p]),
        "gcs_graph_builds": (i32, [P]),
        "gcs_relayout": (C.c_int, [P, i32, C.POINTER(i64), C.POINTER(i32)]),
        "gcs_segment_offset": (i64, [P, i32]),
        "gcs_device_bytes": (i64, [P]),
        "gcs_context_bytes": (i64, [i64, i32, i32]),
        "gcs_bake": (C.c_int, [P, C.POINTER(Params), i32, C.c_char_p, i32, C.POINTER(C.c_double)]),
        "gcs_set_step_range": (C.c_int, [P, i64, i64]),
        "gcs_device_array": (P, [P, i32]),
        "gcs_camera_reference": (None, [C.POINTER(Camera)]),
        "gcs_camera_matrices": (C.c_int, [C.POINTER(Camera), i32, i32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "gcs_camera_look_at": (C.c_int, [C.POINTER(Camera), C.POINTER(C.c_float)]),
        "gcs_render_frame": (C.c_int, [P, C.POINTER(Camera), i32, i32, i32, P, i32]),
        "gcs_render_stars": (C.c_int, [P, i64, C.POINTER(Camera), i32, i32, P, P, P]),
        "gcs_render_playback": (C.c_int, [P, i64, C.POINTER(Camera), i32, i32, P, P, P]),
        "gcs_playback_open": (C.c_int, [C.c_char_p, i64, i64, C.POINTER(P)]),
        "gcs_playback_frames": (i64, [P]),
        "gcs_playback_particles": (i64, [P]),
        "gcs_playback_position": (i64, [P]),
        "gcs_playback_next": (C.c_int, [P, P]),
        "gcs_playback_prev": (C.c_int, [P, P]),
        "gcs_playback_seek": (C.c_int, [P, i64]),
        "gcs_playback_centre": (C.c_int, [P, i64, P]),
        "gcs_playback_close": (None, [P]),
        "gcs_server_create": (C.c_int, [C.POINTER(P), i32, i64, i32, C.c_double, C.POINTER(Params)]),
        "gcs_server_destroy": (None, [P]),
        "gcs_server_context": (P, [P]),
        "gcs_server_capacity": (i64, [P]),
        "gcs_server_last_error": (C.c_char_p, [P]),
        "gcs_server_set_output": (C.c_int, [P, C.c_char_p, i32]),
        "gcs_server_submit": (C.c_int, [P, u64, P, i64, i32]),
        "gcs_server_tick": (C.c_int, [P, C.POINTER(i64)]),
        "gcs_server_counts": (C.c_int, [P, C.POINTER(i64)]),
        "gcs_server_progress": (C.c_int, [P, C.POINTER(i64)]),
        "gcs_server_pop": (C.c_int, [P, C.POINTER(ServerResult), P, i64]),
        "gcs_dropin_set_params": (C.c_int, [C.POINTER(Params)]),
        "gcs_dropin_context": (P, []),
        "gcs_dropin_device_stars": (P, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def reference_params(**kw) -> Params:
    p = Params()
    lib().gcs_params_reference(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def collision_equal(n_disc: int, n_bulge: int, n_halo: int, seed: int = 0) -> np.ndarray:
    """The equal-galaxy recipe (per-galaxy counts given) as a Star array."""
    spec = CollisionSpec()
    _check(lib().gcs_collision_spec_equal(C.byref(spec), n_disc, n_bulge, n_halo, seed), None)
    return _generate(spec)


def collision_pair(n_total: int, q: float, impact: float, rel_speed: float, incline_deg: float,
                   seed: int) -> np.ndarray:
    spec = CollisionSpec()
    _check(lib().gcs_collision_spec_pair(C.byref(spec), n_total, q, impact, rel_speed, incline_deg, seed),
           None)
    return _generate(spec)


def _generate(spec: CollisionSpec) -> np.ndarray:
    n = lib().gcs_collision_count(C.byref(spec))
    out = np.zeros(n, dtype=STAR_DTYPE)
    _check(lib().gcs_generate_collision(C.byref(spec), _ptr(out), n), None)
    return out


def _check(rc: int, ctx) -> None:
    if rc != OK:
        L = lib()
        msg = L.gcs_status_string(rc).decode()
        if ctx is not None:
            msg += ": " + (L.gcs_last_error(ctx) or b"").decode()
        raise GcsError("gcs call failed (%d): %s" % (rc, msg))


# The two configs the recipe names by count.
SMALL_COUNTS = (16384, 4096, 2048)       # 45,056 particles
LARGE_COUNTS = (384000, 96000, 44288)    # 1,048,576 particles


class Context:
    """One gcs_ctx: device state for up to `capacity` particles."""

    def __init__(self, capacity: int, max_segments: int = 1, device: int = 0):
        self._h = C.c_void_p()
        self.L = lib()
        rc = self.L.gcs_create(C.byref(self._h), capacity, max_segments, device)
        if rc != OK:
            raise GcsError("gcs_create failed: %s" % self.L.gcs_status_string(rc).decode())
        self.capacity = capacity

    def close(self) -> None:
        if self._h:
            self.L.gcs_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def check(self, rc: int) -> None:
        _check(rc, self._h)

    def set_stream(self, stream_ptr: int) -> None:
        self.check(self.L.gcs_set_stream(self._h, C.c_void_p(stream_ptr)))

    def set_segments(self, counts) -> None:
        arr = (C.c_int64 * len(counts))(*[int(c) for c in counts])
        self.check(self.L.gcs_set_segments(self._h, len(counts), arr))

    def relayout(self, counts, src_segments) -> None:
        """New layout keeping the device state of segments src_segments[s] >= 0."""
        k = len(counts)
        assert len(src_segments) == k
        c = (C.c_int64 * k)(*[int(x) for x in counts])
        src = (C.c_int32 * k)(*[int(x) for x in src_segments])
        self.check(self.L.gcs_relayout(self._h, k, c, src))

    def segment_offset(self, segment: int) -> int:
        return int(self.L.gcs_segment_offset(self._h, segment))

    @property
    def device_bytes(self) -> int:
        return int(self.L.gcs_device_bytes(self._h))

    @property
    def n(self) -> int:
        return int(self.L.gcs_num_particles(self._h))

    @property
    def n_internal(self) -> int:
        return int(self.L.gcs_num_internal_nodes(self._h))

    def upload(self, stars: np.ndarray, offset: int = 0) -> None:
        stars = np.ascontiguousarray(stars, dtype=STAR_DTYPE)
        self.check(self.L.gcs_upload_stars(self._h, _ptr(stars), offset, len(stars)))

    def download(self, offset: int = 0, n: int | None = None, out: np.ndarray | None = None) -> np.ndarray:
        n = self.n - offset if n is None else n
        out = np.zeros(n, dtype=STAR_DTYPE) if out is None else out
        self.check(self.L.gcs_download_stars(self._h, _ptr(out), offset, n))
        return out

    def download_playback(self, offset: int = 0, n: int | None = None) -> np.ndarray:
        n = self.n - offset if n is None else n
        out = np.zeros(n, dtype=PLAYBACK_DTYPE)
        self.check(self.L.gcs_download_playback(self._h, _ptr(out), offset, n))
        return out

    def step(self, p: Params) -> None:
        self.check(self.L.gcs_step(self._h, C.byref(p)))

    def step_host(self, p: Params, out: np.ndarray) -> None:
        """One step; the stepped Stars (sorted order) land in `out`, copied
        while the walk runs."""
        if out.dtype != STAR_DTYPE or len(out) < self.n or not out.flags.c_contiguous:
            raise ValueError("step_host needs a contiguous Star array of at least n records")
        self.check(self.L.gcs_step_host(self._h, C.byref(p), _ptr(out)))

    def step_host_io(self, p: Params, inp: np.ndarray, out: np.ndarray) -> None:
        """upload(inp) + step_host(p, out) with the upload chunked and
        overlapped with unpacking and the bounds (`out` may be `inp`)."""
        for a in (inp, out):
            if a.dtype != STAR_DTYPE or len(a) < self.n or not a.flags.c_contiguous:
                raise ValueError("step_host_io needs contiguous Star arrays of at least n records")
        self.check(self.L.gcs_step_host_io(self._h, C.byref(p), _ptr(inp), _ptr(out)))

    def compute_accels(self, p: Params) -> None:
        self.check(self.L.gcs_compute_accels(self._h, C.byref(p)))

    def kick(self, dt: float) -> None:
        self.check(self.L.gcs_kick(self._h, dt))

    def run_stages(self, p: Params, first: int, last: int) -> None:
        self.check(self.L.gcs_run_stages(self._h, C.byref(p), first, last))

    def synchronize(self) -> None:
        self.check(self.L.gcs_synchronize(self._h))

    def device_status(self, clear: bool = False) -> int:
        s = C.c_uint32()
        self.check(self.L.gcs_device_status(self._h, C.byref(s), int(clear)))
        return int(s.value)

    _BUF = {BUF_KEYS: ("<u8", 1), BUF_INDEX: ("<u4", 1), BUF_NODES: (NODE_DTYPE, 1),
            BUF_BUILD: (BUILD_DTYPE, 1), BUF_LEAF_PARENT: ("<i4", 1), BUF_ACCEL: ("<f4", 4),
            BUF_POS: ("<f4", 4), BUF_VEL: ("<f4", 4), BUF_BOUNDS: ("<f4", 2),
            BUF_KEYS_UNSORTED: ("<u8", 1)}

    def read(self, which: int, first: int = 0, count: int | None = None) -> np.ndarray:
        dt, width = self._BUF[which]
        if count is None:
            limit = {BUF_NODES: self.n_internal, BUF_BUILD: self.n_internal,
                     BUF_BOUNDS: int(self.L.gcs_num_segments(self._h))}.get(which, self.n)
            count = limit - first
        shape = (count, width) if width > 1 else (count,)
        out = np.zeros(shape, dtype=dt)
        self.check(self.L.gcs_read_buffer(self._h, which, _ptr(out), first, count))
        return out

    def diagnostics(self, segment: int = 0, kick: float = 0.0) -> np.ndarray:
        """{KE, px, py, pz, M, PE} in FP64; velocities taken as v + a * kick."""
        out = (C.c_double * 6)()
        self.check(self.L.gcs_diagnostics_kicked(self._h, segment, kick, out))
        return np.array(out[:])

    def autotune(self, p: Params) -> tuple[Params, float]:
        """Fastest (leaf_size <= p.leaf_size, walk_batch, walk_blocks_per_sm)
        on the current state; the context keeps the fastest group width."""
        q = Params()
        C.memmove(C.byref(q), C.byref(p), C.sizeof(Params))
        ms = C.c_double()
        self.check(self.L.gcs_autotune(self._h, C.byref(q), C.byref(ms)))
        return q, ms.value

    def set_graphs(self, enable: bool) -> None:
        self.check(self.L.gcs_set_graphs(self._h, int(enable)))

    def set_walk_events(self, start, end) -> None:
        """Record two CUDA events (torch.cuda.Event, a raw cudaEvent_t as an
        int, or None) around every walk stage from now on, also inside
        graph-captured steps; see gcs_set_walk_events."""
        def handle(e):
            if e is None:
                return None
            h = getattr(e, "cuda_event", e)
            if not h:
                raise ValueError("the event has no CUDA event yet (record it once first)")
            return C.c_void_p(int(h))
        self.check(self.L.gcs_set_walk_events(self._h, handle(start), handle(end)))

    @property
    def graph_builds(self) -> int:
        return int(self.L.gcs_graph_builds(self._h))

    @property
    def group_width(self) -> int:
        return int(self.L.gcs_group_width(self._h))

    def set_group_width(self, w: int) -> None:
        self.check(self.L.gcs_set_group_width(self._h, w))

    def set_walk_frontier(self, enable: bool) -> None:
        """Super-group frontier pass before the walk (on by default)."""
        self.check(self.L.gcs_set_walk_frontier(self._h, int(bool(enable))))

    def count_interactions(self, p: Params, warp_evals: bool = False):
        """(monopole terms, particle terms)[, warp node evals, warp source evals,
        pop rounds, stack spills, evals opened by all lanes, evals accepted by all]."""
        out = (C.c_uint64 * 8)()
        self.check(self.L.gcs_count_interactions(self._h, C.byref(p), out))
        r = tuple(int(x) for x in out)
        return r if warp_evals else r[:2]

    def walk_lane_use(self) -> dict:
        """Rows the last count_interactions evaluated by kind and the lanes
        (targets) they served; see gcs_walk_lane_use."""
        out = (C.c_uint64 * 8)()
        self.check(self.L.gcs_walk_lane_use(self._h, out))
        keys = ("rows_take_list", "rows_take_full", "rows_take_partial", "rows_mixed",
                "lanes_take_partial", "lanes_mixed", "lanes_mixed_accepting", "lanes_source")
        return dict(zip(keys, (int(x) for x in out)))

    def walk_stack_peak(self):
        """(deepest walk stack of the last count_interactions in entries,
        global-memory stack entries each walk warp may use)."""
        out = (C.c_int64 * 2)()
        self.check(self.L.gcs_walk_stack_peak(self._h, out))
        return int(out[0]), int(out[1])

    def set_step_range(self, first: int, count: int) -> None:
        """Walk and kick/drift only the sorted particles [first, first + count)
        (count < 0: all); see gcs_set_step_range."""
        self.check(self.L.gcs_set_step_range(self._h, first, count))

    def device_array(self, which: int) -> int:
        """Device address of the current POS / VEL / ACCEL array (float4 rows)."""
        ptr = self.L.gcs_device_array(self._h, which)
        if not ptr:
            raise GcsError("gcs_device_array: no such array")
        return int(ptr)

    def device_tensor(self, which: int, torch, rows: int | None = None):
        """A torch float32 tensor [rows, 4] viewing the current POS / VEL /
        ACCEL array in place (no copy); valid until the next step."""
        rows = self.n if rows is None else rows

        class _View:
            pass

        v = _View()
        v.__cuda_array_interface__ = {"shape": (rows, 4), "typestr": "<f4",
                                      "data": (self.device_array(which), False), "version": 3}
        return torch.as_tensor(v, device="cuda")

    def bake(self, p: Params, frames: int, path: str, append: bool = False) -> float:
        """`frames` steps, each written as a simulation.bin frame to `path`;
        returns the wall time in seconds."""
        sec = C.c_double(0.0)
        self.check(self.L.gcs_bake(self._h, C.byref(p), frames, path.encode(), int(append), C.byref(sec)))
        return sec.value

    def render(self, cam: "Camera", width: int, height: int, segment: int = -1) -> np.ndarray:
        """The headless splat frame of the current particles: (height, width, 4)
        uint8 RGBA, row 0 at the bottom (GL's framebuffer order)."""
        out = np.zeros((height, width, 4), np.uint8)
        self.check(self.L.gcs_render_frame(self._h, C.byref(cam), segment, width, height, _ptr(out), 1))
        return out

    def direct_fp64(self, p: Params, targets, segment: int = 0) -> np.ndarray:
        t = np.ascontiguousarray(targets, dtype=np.int64)
        out = np.zeros((len(t), 3), dtype=np.float64)
        self.check(self.L.gcs_direct_accels_fp64(
            self._h, C.byref(p), segment, t.ctypes.data_as(C.POINTER(C.c_int64)), len(t),
            out.ctypes.data_as(C.POINTER(C.c_double))))
        return out


def pos_vel_from_stars(stars: np.ndarray):
    """Split Stars into the engine's (x,y,z,m) and (vx,vy,vz,tcol-bits) float4 rows."""
    n = len(stars)
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    pos[:, 0], pos[:, 1], pos[:, 2], pos[:, 3] = stars["x"], stars["y"], stars["z"], stars["mass"]
    vel[:, 0], vel[:, 1], vel[:, 2] = stars["vx"], stars["vy"], stars["vz"]
    tcol = (stars["type"].astype(np.uint32) | (stars["r"].astype(np.uint32) << 8)
            | (stars["g"].astype(np.uint32) << 16) | (stars["b"].astype(np.uint32) << 24))
    vel[:, 3] = tcol.view(np.float32)
    return pos, vel


def stars_from_pos_vel(pos: np.ndarray, vel: np.ndarray) -> np.ndarray:
    out = np.zeros(len(pos), dtype=STAR_DTYPE)
    out["x"], out["y"], out["z"], out["mass"] = pos[:, 0], pos[:, 1], pos[:, 2], pos[:, 3]
    out["vx"], out["vy"], out["vz"] = vel[:, 0], vel[:, 1], vel[:, 2]
    tcol = np.ascontiguousarray(vel[:, 3]).view(np.uint32)
    out["type"] = tcol & 0xFF
    out["r"] = (tcol >> 8) & 0xFF
    out["g"] = (tcol >> 16) & 0xFF
    out["b"] = (tcol >> 24) & 0xFF
    return out


class Server:
    """Continuous batching of collision scenarios (gcs_server_*)."""

    def __init__(self, p: Params, max_particles: int, max_segments: int, hbm_budget_bytes: float,
                 device: int = 0):
        self.L = lib()
        self._h = C.c_void_p()
        rc = self.L.gcs_server_create(C.byref(self._h), device, max_particles, max_segments,
                                      float(hbm_budget_bytes), C.byref(p))
        if rc != OK:
            raise GcsError("gcs_server_create failed: %s" % self.L.gcs_status_string(rc).decode())
        self._sizes = {}

    def close(self) -> None:
        if self._h:
            self.L.gcs_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int) -> None:
        if rc != OK:
            msg = self.L.gcs_status_string(rc).decode()
            raise GcsError("gcs server call failed (%d): %s: %s" % (
                rc, msg, (self.L.gcs_server_last_error(self._h) or b"").decode()))

    @property
    def capacity(self) -> int:
        return int(self.L.gcs_server_capacity(self._h))

    @property
    def device_bytes(self) -> int:
        return int(self.L.gcs_device_bytes(self.L.gcs_server_context(self._h)))

    def set_output(self, directory: str | None, frame_every: int = 0) -> None:
        d = directory.encode() if directory else None
        self.check(self.L.gcs_server_set_output(self._h, d, frame_every))

    def submit(self, sid: int, stars: np.ndarray, steps: int) -> None:
        stars = np.ascontiguousarray(stars, dtype=STAR_DTYPE)
        self.check(self.L.gcs_server_submit(self._h, sid, _ptr(stars), len(stars), steps))
        self._sizes[sid] = len(stars)

    def tick(self) -> tuple:
        out = (C.c_int64 * 4)()
        self.check(self.L.gcs_server_tick(self._h, out))
        return tuple(int(x) for x in out)

    def counts(self) -> tuple:
        out = (C.c_int64 * 3)()
        self.check(self.L.gcs_server_counts(self._h, out))
        return tuple(int(x) for x in out)

    def progress(self) -> tuple:
        """(particle-steps advanced, steps, peak resident scenarios, peak resident particles)."""
        out = (C.c_int64 * 4)()
        self.check(self.L.gcs_server_progress(self._h, out))
        return tuple(int(x) for x in out)

    def pop(self, with_stars: bool = True):
        """(ServerResult, Stars or None), or None if nothing has finished."""
        info = ServerResult()
        buf = None
        cap = 0
        ptr = None
        if with_stars:
            cap = max(self._sizes.values()) if self._sizes else 0
            buf = np.zeros(cap, dtype=STAR_DTYPE)
            ptr = _ptr(buf)
        rc = self.L.gcs_server_pop(self._h, C.byref(info), ptr, cap)
        if rc == 0:
            return None
        if rc < 0:
            self.check(rc)
        self._sizes.pop(int(info.id), None)
        return info, (buf[:info.n].copy() if with_stars else None)


def context_bytes(capacity: int, max_segments: int = 1, device: int = 0) -> int:
    """Device bytes a Context(capacity, max_segments) would hold."""
    b = int(lib().gcs_context_bytes(capacity, max_segments, device))
    if b < 0:
        _check(b, None)
    return b


def read_playback(path: str, n: int) -> np.ndarray:
    """Frames of a simulation.bin-format file as an array [frames, n] of PlaybackStar."""
    raw = np.fromfile(path, dtype=PLAYBACK_DTYPE)
    if len(raw) % n:
        raise GcsError("%s holds %d records, not a whole number of %d-star frames" % (path, len(raw), n))
    return raw.reshape(-1, n)


class Playback:
    """A simulation.bin file read back frame by frame (gcs_playback_*): the
    reference's Playback mode without its window.  particles > 0 gives the
    records per frame; particles = 0 infers it from frames_hint frames, as
    the reference does with 2000."""

    def __init__(self, path: str, particles: int = 0, frames_hint: int = 2000):
        self.L = lib()
        self._h = C.c_void_p()
        rc = self.L.gcs_playback_open(os.fsencode(path), particles, frames_hint, C.byref(self._h))
        if rc != OK:
            raise GcsError("gcs_playback_open(%s): %s" % (path, self.L.gcs_status_string(rc).decode()))
        self.frames = int(self.L.gcs_playback_frames(self._h))
        self.particles = int(self.L.gcs_playback_particles(self._h))

    def close(self) -> None:
        if self._h:
            self.L.gcs_playback_close(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def position(self) -> int:
        return int(self.L.gcs_playback_position(self._h))

    def _read(self, fn) -> np.ndarray:
        out = np.zeros(self.particles, dtype=PLAYBACK_DTYPE)
        rc = fn(self._h, _ptr(out))
        if rc != OK:
            raise GcsError("playback read: %s" % self.L.gcs_status_string(rc).decode())
        return out

    def next(self) -> np.ndarray:
        return self._read(self.L.gcs_playback_next)

    def prev(self) -> np.ndarray:
        return self._read(self.L.gcs_playback_prev)

    def seek(self, frame: int) -> None:
        _check(self.L.gcs_playback_seek(self._h, frame), None)


def playback_centre(frame: np.ndarray) -> np.ndarray:
    """The reference's per-frame camera target: FP64 mean position as float."""
    frame = np.ascontiguousarray(frame, dtype=PLAYBACK_DTYPE)
    out = np.zeros(3, np.float32)
    _check(lib().gcs_playback_centre(_ptr(frame), len(frame), _ptr(out)), None)
    return out


def camera_reference() -> Camera:
    """The reference's start-up camera (renderer.cpp:9-11, 263)."""
    cam = Camera()
    lib().gcs_camera_reference(C.byref(cam))
    return cam


def camera_look_at(cam: Camera, target) -> Camera:
    """Point cam at target (front = normalize(target - pos)); returns cam."""
    t = (C.c_float * 3)(*[float(x) for x in target])
    rc = lib().gcs_camera_look_at(C.byref(cam), t)
    if rc != OK:
        raise GcsError("gcs_camera_look_at: status %d" % rc)
    return cam


def camera_matrices(cam: Camera, width: int, height: int):
    """(view, proj) 4x4 float32 row-major matrices the renderer uses."""
    v = np.zeros(16, np.float32)
    pm = np.zeros(16, np.float32)
    rc = lib().gcs_camera_matrices(C.byref(cam), width, height, v.ctypes.data_as(C.POINTER(C.c_float)),
                                   pm.ctypes.data_as(C.POINTER(C.c_float)))
    if rc != OK:
        raise GcsError("gcs_camera_matrices: status %d" % rc)
    return v.reshape(4, 4), pm.reshape(4, 4)


def write_ppm(path: str, rgba: np.ndarray) -> None:
    """Write an RGBA frame (row 0 at the bottom) as a binary PPM image (top row first)."""
    h, w = rgba.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(np.ascontiguousarray(rgba[::-1, :, :3]).tobytes())
