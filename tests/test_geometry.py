"""Seeded workload generators: sizes, determinism, the stated definitions."""
import math

import numpy as np

from pawan_b200 import geometry as g


def test_single_ring_defaults():
    sc = g.single_ring()
    assert sc.n == 2048 and sc.nu == 0.0 and sc.dt == 0.01 and sc.steps == 200
    pos, vor, rad, vol = sc.union()
    assert pos.shape == (2048, 3)
    # volume 2 pi R pi sigma^2 / N
    assert np.allclose(vol, 2 * math.pi * math.pi * 0.01 / 2048)
    assert np.allclose(rad, 1.5 * vol ** (1 / 3))
    # per-station strengths sum to Gamma * ds, tangent to the ring
    ds = 2 * math.pi / 256
    st0 = np.linalg.norm(vor[:8], axis=1).sum()
    assert abs(st0 - ds) < 1e-12
    assert abs(np.dot(vor[0], pos[0] / np.linalg.norm(pos[0]))) < 1e-3 * np.linalg.norm(vor[0])


def test_ring_pair_and_helix_sizes():
    assert g.ring_pair(n_stations=8192, steps=1).n == 131072
    h = g.helical_wake(n_stations=64)
    assert h.n == 4 * 64 * 8 and len(h.wakes) == 4


def test_determinism():
    a, b = g.ring_pair(n_stations=16, seed=3), g.ring_pair(n_stations=16, seed=3)
    assert np.array_equal(a.state(), b.state())
    c = g.ring_pair(n_stations=16, seed=4)
    assert not np.array_equal(a.state(), c.state())


def test_jitter_bounds():
    rng = np.random.default_rng(0)
    w = g.ring(1.0, 0.1, 1.0, 32, 0.0, rng)
    w0 = g.ring(1.0, 0.1, 1.0, 32, 0.0, np.random.default_rng(1))
    assert np.abs(w.pos - w0.pos).max() <= 2e-4 + 1e-15


def test_ragged_batch_distribution():
    b = g.ragged_batch(n_solves=64, seed=1)
    ns = np.array([s.n for s in b])
    assert ns.min() >= 512 - 8 and ns.max() <= 16384 + 8 and np.all(ns % 8 == 0)
    assert all(0 <= s.nu <= 1e-3 for s in b)


def test_serving_requests_poisson():
    reqs = g.serving_requests(rate=200, duration=2.0, build=False)
    assert 300 < len(reqs) < 500
    assert all(1024 - 8 <= r.scenario.meta["N"] <= 262144 + 8 for r in reqs)
    assert all(50 <= r.scenario.steps <= 400 for r in reqs)
    t = [r.arrival for r in reqs]
    assert t == sorted(t)
