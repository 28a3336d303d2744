"""Generate the golden vectors in tests/golden/ from the reference's own code.

    python tests/golden/make_golden.py --cpu            # here: morton.h vectors
    python tests/golden/make_golden.py --gpu OUTDIR     # on a B200: reference GPU engine

--cpu runs the reference's morton.h (oracle/_ref/libref_morton.so, built from
the reference sources by oracle/build_ref.py) on seeded inputs and edge cases.
--gpu runs the reference's GPU engine (oracle/_ref/libref_cuda.so: the
reference's cuda_engine.cu/karras_bvh.cuh/CUB, headless, theta as a variable)
on small seeded inputs and records every stage's output; the .npz files it
writes are copied into tests/golden/ and committed.  Inputs are seeded and
built here (no reference files are read at test time).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "galaxy-collision-simulator_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import gcs  # noqa: E402
import oracle  # noqa: E402


def morton_cases():
    rng = np.random.default_rng(1234)
    cases = []
    pts = rng.uniform(-50, 50, size=(4096, 3)).astype(np.float32)
    cases.append(("random", pts, np.float32(pts.min()), np.float32(pts.max())))
    lo, hi = np.float32(-3.25), np.float32(7.5)
    corners = np.array([[x, y, z] for x in (lo, hi) for y in (lo, hi) for z in (lo, hi)], np.float32)
    near = np.array([[np.nextafter(hi, lo)] * 3, [np.nextafter(lo, hi)] * 3, [(lo + hi) / 2] * 3], np.float32)
    cases.append(("corners", np.concatenate([corners, near]), lo, hi))
    tiny = (rng.uniform(0, 1e-3, size=(512, 3)) + 100.0).astype(np.float32)
    cases.append(("tiny_cube", tiny, np.float32(tiny.min()), np.float32(tiny.max())))
    live = rng.normal(0, 300, size=(1024, 3)).astype(np.float32)
    cases.append(("live_bounds", live, np.float32(-10000.0), np.float32(10000.0)))
    grid = (rng.integers(0, 4, size=(1024, 3)) * 0.5).astype(np.float32)
    cases.append(("duplicates", grid, np.float32(grid.min()), np.float32(grid.max())))
    return cases


def make_cpu(outdir: str) -> None:
    L = oracle.ref_lib("ref_morton")
    if L is None:
        raise SystemExit("oracle/_ref/libref_morton.so missing: run oracle/build_ref.py")
    out = {}
    for name, pts, lo, hi in morton_cases():
        xyz = np.ascontiguousarray(pts, np.float32)
        keys = np.zeros(len(xyz), np.uint64)
        L.ref_morton_codes(oracle._ptr(xyz), len(xyz), float(lo), float(hi), oracle._ptr(keys))
        out[name + "_xyz"] = xyz
        out[name + "_lohi"] = np.array([lo, hi], np.float32)
        out[name + "_keys"] = keys
    v = np.array([0, 1, 2, 0x1FFFFF, 0x155555, 0x0AAAAA, 0x100000, 0x3FFFFF, 0xFFFFFFFF], np.uint32)
    out["expand_in"] = v
    out["expand_out"] = np.array([L.ref_expand_bits(int(x)) for x in v], np.uint64)
    np.savez_compressed(os.path.join(outdir, "morton_ref.npz"), **out)
    print("wrote", os.path.join(outdir, "morton_ref.npz"))


# ---- GPU cases ------------------------------------------------------------
def gpu_cases():
    """(name, stars, G, eps2, theta, dt, bounds-or-None)."""
    cases = []
    st = gcs.collision_equal(1024, 256, 128, seed=1)              # 2816 particles
    cases.append(("native_theta1", st, 1.0, 10.0, 1.0, 0.01, None))
    cases.append(("theta05", st, 1.0, 0.05 ** 2, 0.5, 0.005, None))
    rng = np.random.default_rng(7)
    dup = st[:1500].copy()
    g = rng.integers(0, 6, size=(1500, 3)) * 0.75
    dup["x"], dup["y"], dup["z"] = g[:, 0], g[:, 1], g[:, 2]     # heavy key duplication
    cases.append(("duplicates", dup, 1.0, 0.01, 0.7, 0.005, None))
    ref_ic = oracle.ref_initial_conditions(5, 100, 300, 100)      # the reference generator, 1000 particles
    cases.append(("ref_ic_live", ref_ic, 1.0, 10.0, 1.0, 0.01, (-10000.0, 10000.0)))
    return cases


def make_gpu(outdir: str) -> None:
    os.makedirs(outdir, exist_ok=True)
    for name, st, G, eps2, theta, dt, bnd in gpu_cases():
        n = len(st)
        pos, _ = gcs.pos_vel_from_stars(st)
        lo, hi = bnd if bnd is not None else oracle.bounds(pos)
        ref = oracle.RefCuda(n)
        try:
            ref.set_theta(theta)
            ref.upload(st)
            ref.step_device(G, eps2, dt, lo, hi)
            rec = dict(stars=st, params=np.array([G, eps2, theta, dt, lo, hi], np.float32),
                       keys=ref.read(0), perm=ref.read(1), nodes=ref.read(2), build=ref.read(3),
                       accels=ref.read(4), soa=ref.read(5), rgbt=ref.read(6))
        finally:
            ref.close()
        path = os.path.join(outdir, "ref_gpu_%s.npz" % name)
        np.savez_compressed(path, **rec)
        print("wrote", path)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--cpu", action="store_true")
    ap.add_argument("--gpu", metavar="OUTDIR")
    a = ap.parse_args()
    if a.cpu:
        make_cpu(HERE)
    if a.gpu:
        make_gpu(a.gpu)
