"""Shared test setup: import paths, the `gpu` marker, seeded inputs."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "galaxy-collision-simulator_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100) and the built libgcs.so")


@pytest.fixture(scope="session")
def gcs_mod():
    import gcs
    gcs.lib()  # raises if libgcs.so is missing: no silent fallback
    return gcs


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle


def small_collision(n_disc=1024, n_bulge=256, n_halo=128, seed=0):
    import gcs
    return gcs.collision_equal(n_disc, n_bulge, n_halo, seed=seed)


def rel_err(a, b, floor=0.0):
    """Per-row |a-b| / max(|b|, floor)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    num = np.linalg.norm(a - b, axis=-1)
    den = np.maximum(np.linalg.norm(b, axis=-1), floor)
    return num / den
