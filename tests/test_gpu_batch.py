"""Ragged batches: many independent systems in one persistent launch per RK4
stage, with and without CUDA-graph capture."""
import numpy as np
import pytest

import oracle
from pawan_b200 import Batch, PawanError, System, union_to_state
from pawan_b200 import geometry as g
from helpers import TOL_F32_RMS, rms_rel

pytestmark = pytest.mark.gpu


def small_batch(n_solves=7, seed=3):
    return g.ragged_batch(n_solves=n_solves, seed=seed, n_lo=64, n_hi=1500, steps=3)


def test_batch_solve_matches_restatement(ctx):
    scs = small_batch()
    systems = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    b = Batch(ctx, systems)
    b.solve()
    for sc, s in zip(scs, systems):
        pos, vor, rad, vol = sc.union()
        u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, sc.nu)
        u, da = s.union_rates()
        assert rms_rel(u, u_ref) <= TOL_F32_RMS and rms_rel(da, da_ref) <= TOL_F32_RMS


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_rk4_matches_solo_and_restatement(ctx, use_graph):
    scs = small_batch(seed=4)
    systems = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    solos = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    b = Batch(ctx, systems)
    dts = np.array([sc.dt * (1 + 0.1 * k) for k, sc in enumerate(scs)])
    b.rk4(dts, 3, use_graph=use_graph)
    for k, (sc, s, solo) in enumerate(zip(scs, systems, solos)):
        solo.rk4(dts[k], 3)
        st0 = sc.state()
        a, c = s.get_states(), solo.get_states()
        assert rms_rel(a - st0, c - st0) < 1e-12
        pos, vor, rad, vol = sc.union()
        p, v = oracle.rk4_step(pos, vor, rad, vol, sc.nu, dts[k], 3)
        ref = union_to_state(sc.counts, p, v)
        assert rms_rel(a - st0, ref - st0) <= TOL_F32_RMS


def test_gaussian_batch_matches_solo_and_restatement(ctx):
    """Systems with the reference's Gaussian smoothing kernel batched in one
    launch per stage: the same steps as each system alone, and the FP64
    restatement's with that kernel within the FP32 tolerance."""
    scs = small_batch(seed=7)
    systems = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    solos = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    for s in systems + solos:
        s.set_kernel("gaussian")
    b = Batch(ctx, systems)
    b.rk4(scs[0].dt, 2)
    for sc, s, solo in zip(scs, systems, solos):
        solo.rk4(scs[0].dt, 2)
        st0 = sc.state()
        a, c = s.get_states(), solo.get_states()
        assert rms_rel(a - st0, c - st0) < 1e-12
        pos, vor, rad, vol = sc.union()
        p, v = oracle.rk4_step(pos, vor, rad, vol, sc.nu, scs[0].dt, 2, kernel="gaussian")
        ref = union_to_state(sc.counts, p, v)
        assert rms_rel(a - st0, ref - st0) <= TOL_F32_RMS


def test_batch_rejects_mixed_smoothing_kernels(ctx):
    scs = small_batch(n_solves=2, seed=8)
    systems = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    systems[1].set_kernel("gaussian")
    with pytest.raises(PawanError):
        Batch(ctx, systems)


def test_graph_and_eager_agree_bitwise(ctx):
    scs = small_batch(seed=5)
    A = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    B = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    ba, bb = Batch(ctx, A), Batch(ctx, B)
    ba.rk4(0.005, 4, use_graph=True)
    bb.rk4(0.005, 4, use_graph=False)
    for x, y in zip(A, B):
        assert np.array_equal(x.get_states(), y.get_states())


def test_batch_autotune_keeps_results(ctx):
    scs = small_batch(seed=6)
    systems = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    b = Batch(ctx, systems)
    b.autotune()
    b.solve()
    for sc, s in zip(scs, systems):
        pos, vor, rad, vol = sc.union()
        u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, sc.nu)
        u, da = s.union_rates()
        assert rms_rel(u, u_ref) <= TOL_F32_RMS and rms_rel(da, da_ref) <= TOL_F32_RMS


def test_system_autotune(ctx):
    sc = g.single_ring(n_stations=128, seed=2, nu=1e-3)
    s = System.from_scenario(ctx, sc, "f32")
    cfg = s.autotune()
    assert cfg["threads"] in (128, 256) and cfg["threads_per_target"] in (1, 2, 4) and cfg["targets_per_thread"] in (1, 2)
    s.solve()
    pos, vor, rad, vol = sc.union()
    u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, sc.nu)
    u, da = s.union_rates()
    assert rms_rel(u, u_ref) <= TOL_F32_RMS and rms_rel(da, da_ref) <= TOL_F32_RMS
