"""Seeded synthetic wakes with the shapes of the benchmark workloads.

Definitions fixed here (the workload descriptions leave them open):

* A *station* is a cross-section of a vortex tube: one particle on the
  centreline plus ``n_core - 1`` (7) on a circle of radius ``core_frac*sigma``
  (0.5 sigma) in the plane normal to the tube, at angles 2*pi*k/7.
* Core weights ``w ~ exp(-r^2 / (2 sigma^2))``, normalised so that each
  station's weights sum to 1.
* Strength (the reference's "vorticity" alpha, circulation x length) is
  ``Gamma * w_i * ds`` along the tube tangent, ``ds`` the arc length of one
  station -- the same convention as the reference's ``__ring``
  (src/wake/ring.cpp:24-25, strength = gamma*radius*dPsi).
* Volume per particle: tube length * pi * sigma^2 / (particles in the tube);
  for a ring this is 2*pi*R*pi*sigma^2/N.
* Smoothing radius: 1.5 x inter-particle spacing, the spacing taken as
  volume^(1/3).
* Jitter: every coordinate gets uniform(-1e-4, +1e-4) noise from the seeded
  generator (numpy PCG64).

Particles are ordered station-major (index = n_core*station + k).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

N_CORE = 8
CORE_FRAC = 0.5
JITTER = 1e-4
SMOOTHING_FACTOR = 1.5


@dataclass
class Wake:
    """One wake: N particles with position, strength, smoothing radius, volume
    (the fields of the reference's ``__wake``, src/wake/wake.h:33-42)."""
    pos: np.ndarray  # (N, 3) float64
    vor: np.ndarray  # (N, 3) float64
    rad: np.ndarray  # (N,)
    vol: np.ndarray  # (N,)

    @property
    def n(self) -> int:
        return int(self.rad.shape[0])


@dataclass
class Scenario:
    """A system (the reference's ``__interaction``): its wakes and run settings."""
    wakes: List[Wake]
    nu: float
    dt: float
    steps: int
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def counts(self) -> List[int]:
        return [w.n for w in self.wakes]

    @property
    def n(self) -> int:
        return sum(self.counts)

    def union(self):
        """(pos, vor, rad, vol) of all wakes concatenated in wake order."""
        return (np.concatenate([w.pos for w in self.wakes]),
                np.concatenate([w.vor for w in self.wakes]),
                np.concatenate([w.rad for w in self.wakes]),
                np.concatenate([w.vol for w in self.wakes]))

    def state(self) -> np.ndarray:
        """State vector in the reference layout: per wake [x (N x 3) | alpha (N x 3)],
        wakes concatenated (src/wake/wake.cpp:110-120, interaction.cpp:222-229)."""
        return np.concatenate([np.concatenate([w.pos.ravel(), w.vor.ravel()]) for w in self.wakes])

    def wake_ids(self) -> np.ndarray:
        return np.concatenate([np.full(c, i, dtype=np.int32) for i, c in enumerate(self.counts)])


def _core_offsets(sigma: float):
    r = np.zeros(N_CORE)
    ang = np.zeros(N_CORE)
    r[1:] = CORE_FRAC * sigma
    ang[1:] = 2.0 * np.pi * np.arange(N_CORE - 1) / (N_CORE - 1)
    w = np.exp(-r * r / (2.0 * sigma * sigma))
    w /= w.sum()
    return r, ang, w


def _tube(centres, tangents, normals, ds, length, sigma, gamma, rng) -> Wake:
    """Particles of a tube given per-station centre, unit tangent and unit normal."""
    ns = centres.shape[0]
    binormals = np.cross(tangents, normals)
    r, ang, w = _core_offsets(sigma)
    off = (r * np.cos(ang))[None, :, None] * normals[:, None, :] + \
          (r * np.sin(ang))[None, :, None] * binormals[:, None, :]
    pos = (centres[:, None, :] + off).reshape(ns * N_CORE, 3)
    pos = pos + rng.uniform(-JITTER, JITTER, size=pos.shape)
    vor = (gamma * ds * w[None, :, None] * tangents[:, None, :]).reshape(ns * N_CORE, 3)
    n = ns * N_CORE
    volume = length * math.pi * sigma * sigma / n
    rad = np.full(n, SMOOTHING_FACTOR * volume ** (1.0 / 3.0))
    vol = np.full(n, volume)
    return Wake(np.ascontiguousarray(pos), np.ascontiguousarray(vor), rad, vol)


def ring(R: float, sigma: float, gamma: float, n_stations: int, z0: float, rng) -> Wake:
    """Vortex ring of radius R in the plane z = z0, axis +z."""
    th = 2.0 * np.pi * np.arange(n_stations) / n_stations
    c, s = np.cos(th), np.sin(th)
    centres = np.stack([R * c, R * s, np.full_like(th, z0)], axis=1)
    tangents = np.stack([-s, c, np.zeros_like(th)], axis=1)
    normals = np.stack([c, s, np.zeros_like(th)], axis=1)  # radial
    length = 2.0 * np.pi * R
    return _tube(centres, tangents, normals, length / n_stations, length, sigma, gamma, rng)


def helix(R: float, pitch: float, turns: float, phase: float, sigma: float, gamma: float,
          n_stations: int, rng) -> Wake:
    """Helical filament: centre (R cos(t+phase), R sin(t+phase), pitch*t/(2 pi))."""
    t = 2.0 * np.pi * turns * np.arange(n_stations) / n_stations
    a = t + phase
    k = pitch / (2.0 * np.pi)
    centres = np.stack([R * np.cos(a), R * np.sin(a), k * t], axis=1)
    speed = math.sqrt(R * R + k * k)
    tangents = np.stack([-R * np.sin(a), R * np.cos(a), np.full_like(a, k)], axis=1) / speed
    normals = np.stack([-np.cos(a), -np.sin(a), np.zeros_like(a)], axis=1)
    length = speed * 2.0 * np.pi * turns
    return _tube(centres, tangents, normals, length / n_stations, length, sigma, gamma, rng)


# --------------------------------------------------------------- workloads

def single_ring(n_stations: int = 256, seed: int = 1, R: float = 1.0, sigma: float = 0.1,
                gamma: float = 1.0, nu: float = 0.0, dt: float = 0.01, steps: int = 200) -> Scenario:
    """Single vortex ring; defaults are the N=2,048 plain-FP64 workload."""
    rng = np.random.default_rng(seed)
    return Scenario([ring(R, sigma, gamma, n_stations, 0.0, rng)], nu, dt, steps,
                    name=f"single_ring_N{n_stations * N_CORE}", meta={"seed": seed})


def ring_pair(n_stations: int = 8192, seed: int = 2, R: float = 1.0, sigma: float = 0.1,
              gamma: float = 1.0, gap: float = 1.0, nu: float = 1e-4, dt: float = 0.005,
              steps: int = 500) -> Scenario:
    """Leapfrogging coaxial ring pair (two wakes); defaults are N=131,072."""
    rng = np.random.default_rng(seed)
    w1 = ring(R, sigma, gamma, n_stations, 0.0, rng)
    w2 = ring(R, sigma, gamma, n_stations, gap, rng)
    return Scenario([w1, w2], nu, dt, steps, name=f"ring_pair_N{2 * n_stations * N_CORE}",
                    meta={"seed": seed})


def helical_wake(n_stations: int = 8192, seed: int = 3, filaments: int = 4, R: float = 1.0,
                 pitch: float = 0.3, turns: float = 8.0, sigma: float = 0.05, gamma: float = 1.0,
                 nu: float = 1e-3, dt: float = 0.002, steps: int = 300) -> Scenario:
    """Rotor-like wake of helical filaments (one wake each); defaults are N=262,144."""
    rng = np.random.default_rng(seed)
    wakes = [helix(R, pitch, turns, 2.0 * np.pi * f / filaments, sigma, gamma, n_stations, rng)
             for f in range(filaments)]
    return Scenario(wakes, nu, dt, steps, name=f"helical_wake_N{filaments * n_stations * N_CORE}",
                    meta={"seed": seed, "diag_every": 10})


def _log_uniform_n(rng, lo: int, hi: int) -> int:
    n = math.exp(rng.uniform(math.log(lo), math.log(hi)))
    return max(N_CORE, int(round(n / N_CORE)) * N_CORE)


def ragged_batch(n_solves: int = 512, seed: int = 4, n_lo: int = 512, n_hi: int = 16384,
                 dt: float = 0.005, steps: int = 100) -> List[Scenario]:
    """Independent single-ring solves with N log-uniform in [n_lo, n_hi] (rounded
    to whole stations), R~U[0.5,2], sigma/R~U[0.05,0.15], Gamma~U[0.5,2],
    nu~U[0,1e-3]."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_solves):
        n = _log_uniform_n(rng, n_lo, n_hi)
        R = rng.uniform(0.5, 2.0)
        sig = R * rng.uniform(0.05, 0.15)
        gam = rng.uniform(0.5, 2.0)
        nu = rng.uniform(0.0, 1e-3)
        sub = np.random.default_rng([seed, s])
        out.append(Scenario([ring(R, sig, gam, n // N_CORE, 0.0, sub)], nu, dt, steps,
                            name=f"batch{s}_N{n}", meta={"seed": [seed, s]}))
    return out


@dataclass
class Request:
    """One serving request: a single ring or a coaxial ring pair."""
    rid: int
    arrival: float
    scenario: Scenario


def request_wakes(meta: dict) -> List[Wake]:
    """The wakes of a serving request from its drawn parameters (seeded)."""
    sub = np.random.default_rng(meta["seed"])
    n, R, sig, gam = meta["N"], meta["R"], meta["sigma"], meta["gamma"]
    if meta["pair"]:
        per = max(1, n // (2 * N_CORE))
        return [ring(R, sig, gam, per, 0.0, sub), ring(R, sig, gam, per, R, sub)]
    return [ring(R, sig, gam, max(1, n // N_CORE), 0.0, sub)]


def serving_requests(rate: float = 200.0, duration: float = 60.0, seed: int = 5,
                     n_lo: int = 1024, n_hi: int = 262144, steps_lo: int = 50,
                     steps_hi: int = 400, dt: float = 0.005, build: bool = True) -> List[Request]:
    """Poisson arrivals at `rate` per second over `duration` seconds.  With
    build=False only the parameters are drawn (scenario wakes left empty)."""
    rng = np.random.default_rng(seed)
    t, out, rid = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        n = _log_uniform_n(rng, n_lo, n_hi)
        pair = bool(rng.integers(0, 2))
        steps = int(rng.integers(steps_lo, steps_hi + 1))
        R = rng.uniform(0.5, 2.0)
        sig = R * rng.uniform(0.05, 0.15)
        gam = rng.uniform(0.5, 2.0)
        nu = rng.uniform(0.0, 1e-3)
        meta = {"N": n, "pair": pair, "R": R, "sigma": sig, "gamma": gam, "seed": [seed, rid]}
        wakes = request_wakes(meta) if build else []
        out.append(Request(rid, t, Scenario(wakes, nu, dt, steps, name=f"req{rid}", meta=meta)))
        rid += 1
    return out


def expected_n2_loguniform(lo: float, hi: float) -> float:
    """E[N^2] for N log-uniform on [lo, hi]."""
    return (hi * hi - lo * lo) / (2.0 * math.log(hi / lo))
