"""FP64 oracles on the device: the direct sum, the energy/momentum
diagnostics (with and without the leapfrog half-kick) and the walk's
potentials, each against a numpy FP64 restatement on the same snapshot."""
import numpy as np
import pytest

from conftest import small_collision

pytestmark = pytest.mark.gpu


def _params(gcs, **kw):
    p = gcs.reference_params(bounds_mode=gcs.BOUNDS_DEVICE, theta=0.5, epsilon_sq=0.05 ** 2, dt=0.005,
                             leaf_size=4, com_fp64=1)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _direct(pos, G, eps2, targets=None):
    x = pos[:, :3].astype(np.float64)
    m = pos[:, 3].astype(np.float64)
    idx = np.arange(len(x)) if targets is None else np.asarray(targets)
    acc = np.zeros((len(idx), 3))
    phi = np.zeros(len(idx))
    for k, i in enumerate(idx):
        d = x - x[i]
        r2 = np.einsum("ij,ij->i", d, d) + eps2
        inv = 1.0 / np.sqrt(r2)
        inv[i] = 0.0
        acc[k] = G * np.sum((m * inv ** 3)[:, None] * d, axis=0)
        phi[k] = -G * np.sum(m * inv)
    return acc, phi


def test_direct_fp64_matches_numpy(gcs_mod):
    gcs = gcs_mod
    st = small_collision(700, 150, 60, seed=7)
    p = _params(gcs)
    with gcs.Context(len(st)) as ctx:
        ctx.upload(st)
        ctx.compute_accels(p)
        pos = ctx.read(gcs.BUF_POS)
        tg = np.array([0, 1, 17, 500, len(st) - 1])
        got = ctx.direct_fp64(p, tg)
    ref, _ = _direct(pos, p.G, p.epsilon_sq, tg)
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=0)


def test_diagnostics_and_potentials(gcs_mod):
    gcs = gcs_mod
    st = small_collision(500, 120, 40, seed=3)
    n = len(st)
    # theta = 0 opens every node: the walk is a direct sum (FP32 terms)
    p = _params(gcs, theta=0.0, leaf_size=1, with_potential=1)
    with gcs.Context(n) as ctx:
        ctx.upload(st)
        ctx.compute_accels(p)
        pos = ctx.read(gcs.BUF_POS)
        vel = ctx.read(gcs.BUF_VEL)
        acc = ctx.read(gcs.BUF_ACCEL)
        d0 = ctx.diagnostics(0)
        h = 0.0025
        dk = ctx.diagnostics(0, kick=h)
    m = pos[:, 3].astype(np.float64)
    _, phi = _direct(pos, p.G, p.epsilon_sq)
    # potentials of the walk against the FP64 direct sum
    np.testing.assert_allclose(acc[:, 3], phi, rtol=2e-5)
    for out, kick in ((d0, 0.0), (dk, h)):
        v = vel[:, :3].astype(np.float64) + acc[:, :3].astype(np.float64) * kick
        ke = 0.5 * np.sum(m * np.einsum("ij,ij->i", v, v))
        mom = np.sum(m[:, None] * v, axis=0)
        pe = 0.5 * np.sum(m * acc[:, 3].astype(np.float64))
        np.testing.assert_allclose(out[0], ke, rtol=1e-12)
        np.testing.assert_allclose(out[1:4], mom, rtol=1e-10, atol=1e-12 * np.sum(m))
        np.testing.assert_allclose(out[4], np.sum(m), rtol=1e-12)
        np.testing.assert_allclose(out[5], pe, rtol=1e-12)
    assert d0[5] < 0 and abs(dk[0] - d0[0]) > 0


def test_leapfrog_conserves_energy_and_momentum(gcs_mod):
    """A short opened leapfrog run conserves energy to the integrator's
    order and momentum to FP32 rounding of the monopole terms."""
    gcs = gcs_mod
    st = small_collision(2048, 512, 256, seed=1)
    n = len(st)
    dt = 0.005
    p = _params(gcs, dt=dt)
    pp = _params(gcs, dt=dt, with_potential=1)
    with gcs.Context(n) as ctx:
        ctx.upload(st)
        ctx.compute_accels(pp)
        d0 = ctx.diagnostics(0)
        ctx.kick(-0.5 * dt)
        for _ in range(100):
            ctx.step(p)
        ctx.compute_accels(pp)
        d1 = ctx.diagnostics(0, kick=0.5 * dt)
        assert ctx.device_status() == 0
    e0, e1 = d0[0] + d0[5], d1[0] + d1[5]
    assert abs(e1 - e0) / abs(e0) < 2e-3
    v = np.stack([st["vx"], st["vy"], st["vz"]], 1).astype(np.float64)
    scale = np.sum(st["mass"] * np.linalg.norm(v, axis=1))
    assert np.linalg.norm(d1[1:4] - d0[1:4]) / scale < 5e-3


def test_precision_runner_small(gcs_mod, capsys):
    import json
    import precision
    assert precision.main(["--case", "small", "--steps", "20", "--every", "10", "--subset", "512"]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert [r["variant"] for r in out["runs"]] == ["fp64-com", "fp32"]
    for r in out["runs"]:
        assert r["device_status"] == 0
        assert [c["step"] for c in r["checkpoints"]] == [0, 10, 20]
        assert 0 < r["median_force_error"] < 1e-2
        assert r["max_abs_dE_rel"] < 1e-2
