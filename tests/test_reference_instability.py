"""The early blow-up of the ring-pair workload, shown by the reference itself.

The reference's velocity kernel is singular inside the smoothing radius
(q ~ 1/rho^3, src/interaction/highorder.h:57-58).  The leapfrogging ring pair
(8,192 stations per unit ring, smoothing radius 0.022, stations 7.7e-4 apart)
is therefore dominated by its near field: the median particle speed at t = 0 is
about 4 against a ring self-induced speed of about 0.3, and one step of
dt = 0.005 moves particles by tens of station spacings, so the cores scramble
and the strengths grow within a few steps.

Running the reference on all 131,072 particles is out of reach on a CPU, but
the effect is local: the first 128 stations of one of the two rings (N = 1,024,
the same station spacing, core, smoothing radius and volume) show it at t = 0
and over the first six RK4 steps.  Here the reference's own compiled sources
(__parallel with __rk4, OpenMP, oracle/_ref) run that arc, and the project's
FP64 restatement (the checker of the GPU paths) follows the reference over the
first two steps before the chaotic growth separates any two roundings.
CPU only; needs the reference build (make -C oracle).
"""
import numpy as np
import pytest

import oracle
from pawan_b200 import geometry as g
from pawan_b200 import state_to_union

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")

STATIONS = 128


def arc():
    sc = g.ring_pair(steps=1)  # the full workload's first ring, cut to an arc
    w = sc.wakes[0]
    n = g.N_CORE * STATIONS
    return [n], w.pos[:n].copy(), w.vor[:n].copy(), w.rad[:n].copy(), w.vol[:n].copy(), sc.nu, sc.dt


def test_reference_blows_up_on_the_ring_pair_arc():
    counts, pos, vor, rad, vol, nu, dt = arc()
    ref = oracle.RefSystem(counts, pos, vor, rad, vol, nu, parallel=True)
    try:
        ref.solve()
        u0, _ = ref.union_rates()
        speed0 = np.linalg.norm(u0, axis=1)
        # near-field dominated from the start: >= 10x the ring's own speed
        assert np.median(speed0) > 3.0, np.median(speed0)
        state = ref.get_states()
        a0 = np.abs(vor).max()
        growth = []
        prev = (pos, vor)
        for step in range(1, 7):
            state = ref.rk4(state, dt, 1)
            p, v = state_to_union(counts, state)
            growth.append(float(np.abs(v).max() / a0))
            if step <= 2:
                # the restatement follows the reference before the growth sets in
                p1, v1 = oracle.rk4_step(*prev, rad, vol, nu, dt, 1)
                assert np.abs(p1 - p).max() <= 1e-10 * np.abs(p).max()
                assert np.abs(v1 - v).max() <= 1e-8 * np.abs(v).max()
            prev = (p, v)
        # the strengths grow by orders of magnitude within six steps (the
        # reference measured here: 3.7x, 109x, 287x, 1.8e3, 1.1e4, 4.5e4)
        assert growth[-1] > 1e3, growth
        assert max(growth[:2]) < growth[-1]
    finally:
        ref.close()
