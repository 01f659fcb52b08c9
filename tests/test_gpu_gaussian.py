"""The reference's Gaussian smoothing kernel (src/interaction/gaussian.h) on
the GPU, against the reference compiled with it (golden fixtures) and the
oracle restatement: every precision, near and far tiles, mixed radii, RK4,
diagnostics, the vorticity field.  Tolerances as for the default kernel."""
import numpy as np
import pytest

import oracle
from pawan_b200 import System, state_to_union, union_to_state
from pawan_b200 import geometry as g
from helpers import load, max_rel, rms_rel, split_rates, tol

pytestmark = pytest.mark.gpu


def check(prec, u, da, u_ref, da_ref):
    t_rms, t_max = tol(prec)
    assert rms_rel(u, u_ref) <= t_rms and rms_rel(da, da_ref) <= t_rms, (rms_rel(u, u_ref), rms_rel(da, da_ref))
    assert max_rel(u, u_ref) <= t_max and max_rel(da, da_ref) <= t_max, (max_rel(u, u_ref), max_rel(da, da_ref))


def gauss_system(ctx, counts, pos, vor, rad, vol, nu, prec):
    s = System(ctx, counts, nu, prec)
    s.set_kernel("gaussian")
    s.set_particles(pos, vor, rad, vol)
    assert s.kernel == "gaussian"
    return s


@pytest.mark.parametrize("prec", ["f32", "f64", "f64_plain"])
def test_gaussian_matches_golden(ctx, prec):
    d = load("pair64_gauss")
    counts = [int(c) for c in d["counts"]]
    s = gauss_system(ctx, counts, d["pos"], d["vor"], d["rad"], d["vol"], float(d["nu"]), prec)
    s.solve()
    u_ref, da_ref = split_rates(counts, d["rates"])
    check(prec, *s.union_rates(), u_ref, da_ref)
    s.rk4(float(d["dt"]), int(d["nsteps"]))
    inc = s.get_states() - d["state"]
    assert rms_rel(inc, d["final_state"] - d["state"]) <= (1e-5 if prec == "f32" else 1e-10)
    s.set_states(d["state"])
    diag = s.diagnose()
    assert diag["enstrophy"] == 0.0
    assert abs(diag["helicity"] - d["helicity"]) <= 1e-10 * abs(d["helicity"])
    k = s.influence()
    assert rms_rel(k, d["field"]) <= 1e-12


@pytest.mark.parametrize("prec", ["f32", "f64", "f64_plain"])
def test_gaussian_mixed_radii_near_and_far(ctx, prec):
    sc = g.helical_wake(n_stations=64, seed=81, filaments=4, turns=2.0, nu=1e-3)  # N = 2,048
    pos, vor, rad, vol = sc.union()
    rad = rad * np.random.default_rng(8).uniform(0.7, 1.4, rad.shape)
    s = gauss_system(ctx, sc.counts, pos, vor, rad, vol, sc.nu, prec)
    s.solve()
    check(prec, *s.union_rates(), *oracle.pairs(pos, vor, rad, vol, sc.nu, kernel="gaussian"))


@pytest.mark.parametrize("tiling", [(128, 1, 1, 4, 0, 2), (128, 1, 1, 2, 0, 0), (128, 2, 1, 4, 0, 0),
                                    (256, 1, 1, 4, 0, 2)])
def test_gaussian_every_compiled_tiling(ctx, tiling):
    sc = g.ring_pair(n_stations=70, seed=82, nu=1e-3)  # N = 1,120
    pos, vor, rad, vol = sc.union()
    u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, sc.nu, kernel="gaussian")
    s = gauss_system(ctx, sc.counts, pos, vor, rad, vol, sc.nu, "f32")
    tb, p, r, unroll, minb, packed = tiling
    for ips in (1, 16):
        s.set_config(tb, p, unroll, ips, targets_per_thread=r, blocks_per_sm=minb, packed=packed)
        s.solve()
        check("f32", *s.union_rates(), u_ref, da_ref)
    s.autotune()  # only the tilings compiled for this kernel are candidates
    s.solve()
    check("f32", *s.union_rates(), u_ref, da_ref)


def test_gaussian_rk4_matches_oracle_and_switching_back(ctx):
    sc = g.single_ring(n_stations=64, seed=83, nu=2e-3)
    pos, vor, rad, vol = sc.union()
    s = gauss_system(ctx, sc.counts, pos, vor, rad, vol, sc.nu, "f32")
    s.rk4(sc.dt, 3)
    p1, v1 = oracle.rk4_step(pos, vor, rad, vol, sc.nu, sc.dt, 3, kernel="gaussian")
    ref = union_to_state(sc.counts, p1, v1)
    st0 = sc.state()
    assert rms_rel(s.get_states() - st0, ref - st0) <= 1e-5
    s.set_kernel("highorder")
    s.set_states(st0)
    s.solve()
    check("f32", *s.union_rates(), *oracle.pairs(pos, vor, rad, vol, sc.nu))


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("gap", [6.0, 7.5, 10.0])
def test_gaussian_far_class_at_its_boundary(ctx, gap, mixed):
    """Two compact clusters of 256 particles whose boxes are `gap` smoothing
    radii apart: below 7 sigma the Gaussian far tiles evaluate exp and erf,
    from 7 sigma on (8.4 s with radii in [0.8 s, 1.2 s]) the singular field
    they equal there to FP32 resolution.  The cross-cluster part at cluster A
    on its own (by linearity: B's strengths doubled, minus the first solve)
    against the same difference in the FP64 oracle, on every compiled
    Gaussian tiling; B's strengths share a direction so that the part is well
    conditioned."""
    rng = np.random.default_rng(int(gap * 10) + 1)
    s = 0.05
    n = 256
    a = rng.uniform(-0.5 * s, 0.5 * s, (n, 3))
    b = rng.uniform(-0.5 * s, 0.5 * s, (n, 3))
    b[:, 0] += (gap + 1.0) * s  # box gap = gap * s
    pos = np.concatenate([a, b])
    vor = rng.normal(size=(2 * n, 3)) * 1e-3
    vor[n:] += np.array([1e-3, 2e-3, -1.5e-3])
    vor2 = vor.copy()
    vor2[n:] *= 2.0
    rad = s * rng.uniform(0.8, 1.2, 2 * n) if mixed else np.full(2 * n, s)
    vol = np.full(2 * n, 1e-5)
    nu = 1e-3
    u1, da1 = oracle.pairs(pos, vor, rad, vol, nu, kernel="gaussian")
    u2, da2 = oracle.pairs(pos, vor2, rad, vol, nu, kernel="gaussian")
    du_ref, dda_ref = (u2 - u1)[:n], (da2 - da1)[:n]
    st1, st2 = union_to_state([2 * n], pos, vor), union_to_state([2 * n], pos, vor2)
    sysm = gauss_system(ctx, [2 * n], pos, vor, rad, vol, nu, "f32")
    for tb, p, r, unroll, minb, packed in [(128, 1, 1, 4, 0, 2), (128, 1, 1, 2, 0, 0), (128, 2, 1, 4, 0, 0),
                                          (256, 1, 1, 4, 0, 2)]:
        sysm.set_config(tb, p, unroll, 16, targets_per_thread=r, blocks_per_sm=minb, packed=packed)
        sysm.set_states(st1)
        sysm.solve()
        ug1, dag1 = sysm.union_rates()
        check("f32", ug1, dag1, u1, da1)
        sysm.set_states(st2)
        sysm.solve()
        ug2, dag2 = sysm.union_rates()
        du, dda = (ug2 - ug1)[:n], (dag2 - dag1)[:n]
        assert rms_rel(du, du_ref) < 1e-5 and rms_rel(dda, dda_ref) < 1e-5, \
            (tb, p, packed, rms_rel(du, du_ref), rms_rel(dda, dda_ref))


@pytest.mark.parametrize("tiling", [(256, 1, 1, 4, 0, 2), (128, 1, 1, 2, 0, 0)])
def test_gaussian_full_size_sampled_targets(ctx, tiling):
    """The ring pair at full size (N = 131,072) with the Gaussian kernel, where
    nearly every tile pair takes the far class: 4,096 sampled targets against
    the FP64 restatement summed over all N sources, packed and scalar far
    loops."""
    sc = g.ring_pair(steps=1)
    pos, vor, rad, vol = sc.union()
    t = np.sort(np.random.default_rng(1).choice(sc.n, 4096, replace=False))
    u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, sc.nu, targets=t, kernel="gaussian")
    s = gauss_system(ctx, sc.counts, pos, vor, rad, vol, sc.nu, "f32")
    tb, p, r, unroll, minb, packed = tiling
    s.set_config(tb, p, unroll, 64, targets_per_thread=r, blocks_per_sm=minb, packed=packed)
    s.solve()
    u, da = s.union_rates()
    check("f32", u[t], da[t], u_ref, da_ref)
