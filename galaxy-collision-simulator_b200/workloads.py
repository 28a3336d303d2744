"""Seeded scenario streams for the batched and served workloads.

* batched: independent two-galaxy collisions with particle counts drawn
  log-uniform in [4,096, 262,144], mass ratio uniform in [0.2, 1], impact
  parameter uniform in [0, 15], disc inclination uniform in [0, 90] degrees
  and relative speed uniform in [0.3, 0.8]; scenario i uses IC seed i.
* served: requests arriving as a Poisson process of a given rate, with N
  log-uniform in [8,192, 1,048,576], step counts uniform in [100, 2,000] and
  the other parameters drawn as in the batched stream.

The reference simulates one hard-coded scenario per process (main.cpp:28-34);
these streams exist to load the segmented engine and the server.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Scenario:
    index: int
    n: int
    q: float
    impact: float
    incline_deg: float
    rel_speed: float
    seed: int
    steps: int = 0
    arrival_s: float = 0.0

    def stars(self, gcs):
        return gcs.collision_pair(self.n, self.q, self.impact, self.rel_speed, self.incline_deg, self.seed)


def _log_uniform(rng, lo, hi):
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def _draw(rng, i, n_lo, n_hi):
    n = _log_uniform(rng, n_lo, n_hi)
    q = float(rng.uniform(0.2, 1.0))
    impact = float(rng.uniform(0.0, 15.0))
    incline = float(rng.uniform(0.0, 90.0))
    speed = float(rng.uniform(0.3, 0.8))
    return Scenario(index=i, n=n, q=q, impact=impact, incline_deg=incline, rel_speed=speed, seed=i)


def batched_scenarios(count: int = 256, n_lo: int = 4096, n_hi: int = 262144, steps: int = 500,
                      seed: int = 0) -> list[Scenario]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        s = _draw(rng, i, n_lo, n_hi)
        s.steps = steps
        out.append(s)
    return out


def serving_requests(count: int, rate_per_s: float, seed: int = 0, n_lo: int = 8192, n_hi: int = 1 << 20,
                     steps_lo: int = 100, steps_hi: int = 2000, step_scale: float = 1.0) -> list[Scenario]:
    """`count` requests; arrival times are cumulative exponential gaps of mean
    1/rate_per_s.  step_scale shortens every request's step count (at least 1
    step) to bound the run time; it is reported beside any number measured."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        s = _draw(rng, i, n_lo, n_hi)
        steps = int(rng.integers(steps_lo, steps_hi + 1))
        s.steps = max(1, int(round(steps * step_scale)))
        t += float(rng.exponential(1.0 / rate_per_s))
        s.arrival_s = t
        out.append(s)
    return out
