"""Accuracy and conservation runs of the Barnes-Hut step.

    python galaxy-collision-simulator_b200/precision.py --case large   # 1,048,576 particles
    python galaxy-collision-simulator_b200/precision.py --case precision  # 4,194,304 particles

For each variant the scenario is integrated with the leapfrog: the stored
velocities are half-step ones (the reference's update v += a dt; x += v dt,
cuda_engine.cu:164-216, is the leapfrog in that form), opened from the
synchronised initial velocities by a half-kick v_{-1/2} = v_0 - a_0 dt/2.
Every `every` steps the accelerations and potentials are computed at the
current positions and the run records
  * the relative force error |a_BH - a_exact| / |a_exact| against an FP64
    direct sum (excluding only i == j) on a seeded random subset of targets
    (median and 99th percentile);
  * total energy KE + PE (FP64 sums; KE at the synchronised velocities
    v_n = v_{n-1/2} + a_n dt/2, PE = 1/2 sum m phi from the walk's
    potentials) and linear momentum, whose drifts are reported relative to
    |E_0| and to sum m |v_0|.

Variants: "fp64-com" keeps FP64 only where it is needed (node centre-of-mass
sums and the diagnostics); "fp32" is all-FP32 (the reference's pairwise FP32
centre of mass).  Morton bounds are exact min/max reductions in both.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import gcs  # noqa: E402

CASES = {
    # two equal galaxies (2 x [384,000 disc + 96,000 bulge + 44,288 halo])
    "large": dict(recipe="equal", counts=(384000, 96000, 44288), theta=[0.5, 0.7], eps=0.02, dt=0.0025,
                  steps=1000, every=100, variants=["fp64-com"]),
    # 1:3 mass ratio, impact parameter 8, relative speed 0.6
    "precision": dict(recipe="pair", n=4194304, q=1.0 / 3.0, impact=8.0, speed=0.6, incline=30.0,
                      theta=[0.5], eps=0.01, dt=0.002, steps=2000, every=100, variants=["fp64-com", "fp32"]),
    # the 45,056-particle case, for a quick check
    "small": dict(recipe="equal", counts=(16384, 4096, 2048), theta=[0.5], eps=0.05, dt=0.005, steps=200,
                  every=50, variants=["fp64-com", "fp32"]),
}


def initial_stars(case: dict, seed: int) -> np.ndarray:
    if case["recipe"] == "equal":
        return gcs.collision_equal(*case["counts"], seed=seed)
    return gcs.collision_pair(case["n"], case["q"], case["impact"], case["speed"], case["incline"], seed)


def force_error(ctx, p, n, subset, rng) -> dict:
    acc = ctx.read(gcs.BUF_ACCEL)[:, :3].astype(np.float64)
    tg = np.sort(rng.choice(n, size=min(subset, n), replace=False))
    exact = ctx.direct_fp64(p, tg)
    e = np.linalg.norm(acc[tg] - exact, axis=1) / np.linalg.norm(exact, axis=1)
    return {"median": float(np.median(e)), "p99": float(np.percentile(e, 99)), "max": float(e.max())}


def run_variant(stars, theta, eps, dt, steps, every, leaf, com_fp64, subset, seed, stream_ptr):
    n = len(stars)
    p = gcs.reference_params(theta=theta, epsilon_sq=eps * eps, dt=dt, leaf_size=leaf,
                             bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=com_fp64, recolor=1)
    pp = gcs.reference_params(theta=theta, epsilon_sq=eps * eps, dt=dt, leaf_size=leaf,
                              bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=com_fp64, recolor=1, with_potential=1)
    rng = np.random.default_rng(seed)
    rows = []
    t0 = time.perf_counter()
    with gcs.Context(n) as ctx:
        if stream_ptr:
            ctx.set_stream(stream_ptr)
            ctx.set_graphs(True)
        ctx.upload(stars)

        def checkpoint(step, kick):
            ctx.compute_accels(pp)
            d = ctx.diagnostics(0, kick=kick)
            row = {"step": step, "KE": d[0], "PE": d[5], "E": d[0] + d[5], "P": [d[1], d[2], d[3]]}
            row["force_error"] = force_error(ctx, p, n, subset, rng)
            rows.append(row)

        checkpoint(0, 0.0)
        d0 = ctx.diagnostics(0, kick=0.0)
        v = np.stack([stars["vx"], stars["vy"], stars["vz"]], 1).astype(np.float64)
        p_scale = float(np.sum(stars["mass"].astype(np.float64) * np.linalg.norm(v, axis=1)))
        ctx.kick(-0.5 * dt)  # open the leapfrog: half-step velocities
        for k in range(1, steps + 1):
            ctx.step(p)
            if k % every == 0 or k == steps:
                checkpoint(k, 0.5 * dt)
        status = ctx.device_status()
    wall = time.perf_counter() - t0
    e0 = rows[0]["E"]
    p0 = np.array(rows[0]["P"])
    for r in rows:
        r["dE_rel"] = (r["E"] - e0) / abs(e0)
        r["dP_rel"] = float(np.linalg.norm(np.array(r["P"]) - p0) / p_scale)
    return {"theta": theta, "eps": eps, "dt": dt, "steps": steps, "leaf_size": leaf, "com_fp64": com_fp64,
            "particles": n, "mass": float(d0[4]), "device_status": status, "wall_s": wall,
            "max_abs_dE_rel": max(abs(r["dE_rel"]) for r in rows), "final_dE_rel": rows[-1]["dE_rel"],
            "max_dP_rel": max(r["dP_rel"] for r in rows),
            "median_force_error": float(np.median([r["force_error"]["median"] for r in rows])),
            "p99_force_error": float(np.median([r["force_error"]["p99"] for r in rows])),
            "checkpoints": rows}


def com_effect(stars, theta, eps, leaf) -> dict:
    """Accelerations on the initial snapshot with FP64 and with FP32 node
    centres of mass: relative difference per particle (same tree, same
    walk), i.e. what the FP64 sums change."""
    n = len(stars)
    out = {}
    with gcs.Context(n) as ctx:
        acc = []
        for com in (1, 0):
            p = gcs.reference_params(theta=theta, epsilon_sq=eps * eps, leaf_size=leaf,
                                     bounds_mode=gcs.BOUNDS_DEVICE, com_fp64=com)
            ctx.upload(stars)
            ctx.compute_accels(p)
            acc.append(ctx.read(gcs.BUF_ACCEL)[:, :3].astype(np.float64))
        d = np.linalg.norm(acc[0] - acc[1], axis=1) / np.linalg.norm(acc[0], axis=1)
        out = {"median": float(np.median(d)), "p99": float(np.percentile(d, 99)), "max": float(d.max())}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=sorted(CASES), default="small")
    ap.add_argument("--steps", type=int, default=0, help="override the case's step count")
    ap.add_argument("--every", type=int, default=0, help="override the checkpoint interval")
    ap.add_argument("--leaf", type=int, default=4)
    ap.add_argument("--subset", type=int, default=65536)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default="", help="write the JSON here as well")
    args = ap.parse_args(argv)
    case = dict(CASES[args.case])
    steps = args.steps or case["steps"]
    every = args.every or case["every"]
    import torch  # noqa: PLC0415  (a non-default stream for the step graphs)
    stream = torch.cuda.Stream()
    stars = initial_stars(case, args.seed)
    out = {"case": args.case, "particles": len(stars), "seed": args.seed, "subset": args.subset, "runs": []}
    out["fp64_vs_fp32_com_accel_rel_diff"] = com_effect(stars, case["theta"][0], case["eps"], args.leaf)
    for theta in case["theta"]:
        for var in case["variants"]:
            r = run_variant(stars, theta, case["eps"], case["dt"], steps, every, args.leaf,
                            1 if var == "fp64-com" else 0, args.subset, args.seed, stream.cuda_stream)
            r["variant"] = var
            out["runs"].append(r)
            print("%s theta=%.2f %s: force error median %.3e p99 %.3e | max |dE/E| %.3e | max dP %.3e | %.1f s"
                  % (args.case, theta, var, r["median_force_error"], r["p99_force_error"], r["max_abs_dE_rel"],
                     r["max_dP_rel"], r["wall_s"]), file=sys.stderr)
    text = json.dumps(out)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text + "\n")
    print(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
