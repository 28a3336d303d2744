"""ctypes binding of the oracle: the C restatement (liboracle.so) and the
reference's own code compiled by build_ref.py (oracle/_ref/*.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the engine.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "galaxy-collision-simulator_b200"))
from gcs import NODE_DTYPE, STAR_DTYPE  # noqa: E402

_P = C.c_void_p
_i32, _i64, _u32, _u64, _f32, _f64 = C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_float, C.c_double
_o = None


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def lib() -> C.CDLL:
    global _o
    if _o is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            from build_ref import build_oracle  # noqa: PLC0415
            build_oracle()
        L = C.CDLL(path)
        sig = {
            "gcs_oracle_f2u_rz": (_u32, [_f32]),
            "gcs_oracle_spread21": (_u64, [_u32]),
            "gcs_oracle_morton": (_u64, [_f32, _f32, _f32, _f32, _f32]),
            "gcs_oracle_encode": (None, [_P, _i64, _f32, _f32, _P]),
            "gcs_oracle_bounds": (None, [_P, _i64, C.POINTER(_f32), C.POINTER(_f32)]),
            "gcs_oracle_sort": (None, [_P, _i64, _P, _P]),
            "gcs_oracle_build": (None, [_P, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P]),
            "gcs_oracle_aggregate": (None, [C.c_int, _P, _P, _P, C.c_int]),
            "gcs_oracle_walk": (None, [C.c_int, _P, _P, _f32, _f32, _f32, C.c_int, _P, _P]),
            "gcs_oracle_integrate": (None, [_i64, _P, _P, _P, _f32, C.c_int]),
            "gcs_oracle_render": (None, [_P, _i64, _P, _P, C.c_int, C.c_int, _P, _P]),
            "gcs_oracle_walk_targets": (None, [C.c_int, _P, _P, _f32, _f32, _f32, C.c_int, _P, _i64, _P, _P]),
            "gcs_oracle_direct_fp64": (None, [_i64, _P, _P, _i64, _f64, _f64, _P]),
            "gcs_oracle_step": (None, [C.c_int, _P, _P, C.c_int, _f32, _f32, _f32, _f32, _f32, C.c_int,
                                       _f32, C.c_int, C.c_int, _P, _P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _o = L
    return _o


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def bounds(xyzm: np.ndarray):
    lo, hi = _f32(), _f32()
    x = f32(xyzm)
    lib().gcs_oracle_bounds(_ptr(x), len(x), C.byref(lo), C.byref(hi))
    return np.float32(lo.value), np.float32(hi.value)


def encode(xyzm: np.ndarray, lo: float, hi: float) -> np.ndarray:
    x = f32(xyzm)
    keys = np.zeros(len(x), np.uint64)
    lib().gcs_oracle_encode(_ptr(x), len(x), lo, hi, _ptr(keys))
    return keys


def sort(keys: np.ndarray):
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    ko = np.zeros_like(k)
    io = np.zeros(len(k), np.uint32)
    lib().gcs_oracle_sort(_ptr(k), len(k), _ptr(ko), _ptr(io))
    return ko, io


def build(sorted_keys: np.ndarray, node_base: int = 0, leaf_base: int | None = None, off: int = 0):
    """Karras tree of one segment -> (child_left, child_right, range_end, parent, leaf_parent)."""
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint64)
    n = len(k)
    leaf_base = n - 1 if leaf_base is None else leaf_base
    m = max(n - 1, 1)
    cl, cr, re, par = (np.zeros(m, np.int32) for _ in range(4))
    lp = np.zeros(n, np.int32)
    lib().gcs_oracle_build(_ptr(k), n, node_base, leaf_base, off, _ptr(cl), _ptr(cr), _ptr(re), _ptr(par), _ptr(lp))
    return cl[: n - 1], cr[: n - 1], re[: n - 1], par[: n - 1], lp


def aggregate(xyzm: np.ndarray, cl, cr, re, com_fp64: bool = False):
    """Fill the node records of one segment's tree -> (nodes, box[n-1,6])."""
    x = f32(xyzm)
    n = len(x)
    nodes = np.zeros(max(n - 1, 1), NODE_DTYPE)
    nodes["child_left"][: n - 1] = cl
    nodes["child_right"][: n - 1] = cr
    nodes["range_end"][: n - 1] = re
    box = np.zeros((max(n - 1, 1), 6), np.float32)
    lib().gcs_oracle_aggregate(n, _ptr(x), _ptr(nodes), _ptr(box), int(com_fp64))
    return nodes[: n - 1], box[: n - 1]


def walk(xyzm: np.ndarray, nodes: np.ndarray, G: float, eps2: float, theta: float, leaf_size: int,
         counts: bool = False):
    x = f32(xyzm)
    n = len(x)
    nd = np.ascontiguousarray(nodes, dtype=NODE_DTYPE)
    if len(nd) == 0:
        nd = np.zeros(1, NODE_DTYPE)
    acc = np.zeros((n, 4), np.float32)
    cnt = np.zeros((n, 2), np.int64) if counts else None
    lib().gcs_oracle_walk(n, _ptr(x), _ptr(nd), G, eps2, theta, leaf_size, _ptr(acc),
                          _ptr(cnt) if counts else None)
    return (acc, cnt) if counts else acc


def walk_targets(xyzm: np.ndarray, nodes: np.ndarray, G: float, eps2: float, theta: float, leaf_size: int,
                 targets) -> tuple:
    """walk() for the listed targets only -> (acc [k, 4], counts [k, 2])."""
    x = f32(xyzm)
    nd = np.ascontiguousarray(nodes, dtype=NODE_DTYPE)
    if len(nd) == 0:
        nd = np.zeros(1, NODE_DTYPE)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    acc = np.zeros((len(t), 4), np.float32)
    cnt = np.zeros((len(t), 2), np.int64)
    lib().gcs_oracle_walk_targets(len(x), _ptr(x), _ptr(nd), G, eps2, theta, leaf_size, _ptr(t), len(t), _ptr(acc),
                                  _ptr(cnt))
    return acc, cnt


def integrate(xyzm: np.ndarray, vel4: np.ndarray, acc4: np.ndarray, dt: float, recolor: bool = True):
    x = f32(xyzm).copy()
    v = f32(vel4).copy()
    a = f32(acc4)
    lib().gcs_oracle_integrate(len(x), _ptr(x), _ptr(v), _ptr(a), dt, int(recolor))
    return x, v


def direct_fp64(xyzm: np.ndarray, targets, G: float, eps2: float) -> np.ndarray:
    x = f32(xyzm)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros((len(t), 3), np.float64)
    lib().gcs_oracle_direct_fp64(len(x), _ptr(x), _ptr(t), len(t), G, eps2, _ptr(out))
    return out


def step(xyzm, vel4, G, eps2, theta, leaf_size, dt, bounds_lohi=None, recolor=True, com_fp64=False):
    """One reference step of one segment -> (xyzm', vel4', acc, nodes), all in sorted order."""
    x = f32(xyzm).copy()
    v = f32(vel4).copy()
    n = len(x)
    acc = np.zeros((n, 4), np.float32)
    nodes = np.zeros(max(n - 1, 1), NODE_DTYPE)
    use = bounds_lohi is not None
    lo, hi = bounds_lohi if use else (0.0, 0.0)
    lib().gcs_oracle_step(n, _ptr(x), _ptr(v), int(use), lo, hi, G, eps2, theta, leaf_size, dt, int(recolor),
                          int(com_fp64), _ptr(acc), _ptr(nodes))
    return x, v, acc, nodes[: n - 1]


def render(stars: np.ndarray, view: np.ndarray, proj: np.ndarray, width: int, height: int):
    """CPU restatement of the splat renderer -> (acc uint64 [h, w, 3], rgba uint8 [h, w, 4])."""
    st = np.ascontiguousarray(stars)
    assert st.dtype.itemsize == 32
    v = f32(np.asarray(view).ravel())
    p = f32(np.asarray(proj).ravel())
    acc = np.zeros((height, width, 3), np.uint64)
    rgba = np.zeros((height, width, 4), np.uint8)
    lib().gcs_oracle_render(_ptr(st), len(st), _ptr(v), _ptr(p), width, height, _ptr(acc), _ptr(rgba))
    return acc, rgba


# ---------------------------------------------------------------------------
# The reference's own code (oracle/_ref), when it was built.
# ---------------------------------------------------------------------------
def ref_lib(name: str):
    """Load oracle/_ref/lib<name>.so or return None if it was not built."""
    path = os.path.join(REF_DIR, "lib%s.so" % name)
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    if name == "ref_morton":
        L.ref_morton_codes.argtypes = [_P, _i64, _f32, _f32, _P]
        L.ref_morton_codes.restype = None
        L.ref_expand_bits.argtypes = [_u32]
        L.ref_expand_bits.restype = _u64
    elif name == "ref_cpu":
        L.ref_cpu_init.argtypes = [_i64, _i64]
        L.ref_cpu_init.restype = C.c_int
        L.ref_cpu_cleanup.argtypes = []
        L.ref_cpu_set_theta.argtypes = [_f32]
        L.ref_cpu_threads.restype = C.c_int
        L.ref_cpu_step.argtypes = [_P, C.c_int, _f32, _f32, _f32, _P, _P]
        L.ref_cpu_step.restype = C.c_int
        L.ref_initial_setup.argtypes = [_u32, C.c_int, C.c_int, C.c_int, _P]
        L.ref_initial_setup.restype = None
    elif name == "ref_cuda":
        L.ref_cuda_init.argtypes = [C.c_int]
        L.ref_cuda_init.restype = C.c_int
        L.ref_cuda_cleanup.argtypes = []
        L.ref_cuda_upload.argtypes = [_P, C.c_int]
        L.ref_cuda_set_theta.argtypes = [_f32]
        L.ref_cuda_set_theta.restype = C.c_int
        L.ref_cuda_step.argtypes = [_P, C.c_int, _f32, _f32, _f32, _f32, _f32]
        L.ref_cuda_step.restype = _f32
        L.ref_cuda_step_device.argtypes = [C.c_int, _f32, _f32, _f32, _f32, _f32]
        L.ref_cuda_step_device.restype = _f32
        L.ref_cuda_time_walk.argtypes = [C.c_int, _f32, _f32]
        L.ref_cuda_time_walk.restype = _f32
        L.ref_cuda_read.argtypes = [C.c_int, _P, C.c_int]
        L.ref_cuda_read.restype = C.c_int
    return L


def collision_equal(n_disc: int, n_bulge: int, n_halo: int, seed: int = 0) -> np.ndarray:
    """The equal-galaxy recipe's seeded initial conditions from
    oracle/_ref/libic.so (the same generator source as the engine library's
    gcs.collision_equal, built on its own so a caller need not load the
    engine)."""
    from gcs import CollisionSpec  # noqa: PLC0415  (ctypes layout only; loads no library)
    path = os.path.join(REF_DIR, "libic.so")
    if not os.path.exists(path):
        from build_ref import build_ic  # noqa: PLC0415
        build_ic()
    L = C.CDLL(path)
    L.gcs_collision_spec_equal.argtypes = [C.POINTER(CollisionSpec), _i64, _i64, _i64, _u64]
    L.gcs_collision_spec_equal.restype = C.c_int
    L.gcs_collision_count.argtypes = [C.POINTER(CollisionSpec)]
    L.gcs_collision_count.restype = _i64
    L.gcs_generate_collision.argtypes = [C.POINTER(CollisionSpec), _P, _i64]
    L.gcs_generate_collision.restype = C.c_int
    spec = CollisionSpec()
    if L.gcs_collision_spec_equal(C.byref(spec), n_disc, n_bulge, n_halo, seed) != 0:
        raise RuntimeError("collision spec rejected")
    n = L.gcs_collision_count(C.byref(spec))
    out = np.zeros(n, STAR_DTYPE)
    if L.gcs_generate_collision(C.byref(spec), _ptr(out), n) != 0:
        raise RuntimeError("initial-conditions generator failed")
    return out


def ref_initial_conditions(seed: int, num_dm: int, num_disc: int, num_bulge: int) -> np.ndarray:
    """The reference generator's own two-galaxy setup (generator.cpp:169-210), seeded."""
    L = ref_lib("ref_cpu")
    if L is None:
        raise RuntimeError("oracle/_ref/libref_cpu.so not built")
    out = np.zeros(2 * (num_dm + num_disc + num_bulge), STAR_DTYPE)
    L.ref_initial_setup(seed, num_dm, num_disc, num_bulge, _ptr(out))
    return out


class RefCuda:
    """The reference GPU engine (one process-wide instance, like the original)."""

    def __init__(self, n: int):
        self.L = ref_lib("ref_cuda")
        if self.L is None:
            raise RuntimeError("oracle/_ref/libref_cuda.so not built")
        if self.L.ref_cuda_init(n) != 0:
            raise RuntimeError("reference cuda_init failed")
        self.n = n

    def close(self):
        if self.L is not None:
            self.L.ref_cuda_cleanup()
            self.L = None

    def upload(self, stars: np.ndarray):
        s = np.ascontiguousarray(stars, STAR_DTYPE)
        self.L.ref_cuda_upload(_ptr(s), len(s))

    def set_theta(self, theta: float):
        assert self.L.ref_cuda_set_theta(theta) == 0

    def step_device(self, G, eps2, dt, lo, hi) -> float:
        return float(self.L.ref_cuda_step_device(self.n, G, eps2, dt, lo, hi))

    def step(self, out: np.ndarray, G, eps2, dt, lo, hi) -> float:
        return float(self.L.ref_cuda_step(_ptr(out), self.n, G, eps2, dt, lo, hi))

    def time_walk(self, G, eps2) -> float:
        return float(self.L.ref_cuda_time_walk(self.n, G, eps2))

    def read(self, which: int) -> np.ndarray:
        n = self.n
        shapes = {0: (np.uint64, (n,)), 1: (np.int32, (n,)), 2: (NODE_DTYPE, (2 * n - 1,)),
                  3: (np.dtype([("min", "<f4", 3), ("max", "<f4", 3), ("flag", "<i4"), ("parent", "<i4")]),
                      (2 * n - 1,)),
                  4: (np.float32, (n, 3)), 5: (np.float32, (7, n)), 6: (np.uint8, (4, n))}
        dt, shape = shapes[which]
        out = np.zeros(shape, dt)
        assert self.L.ref_cuda_read(which, _ptr(out), n) == 0
        return out
