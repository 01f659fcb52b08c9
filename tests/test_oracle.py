"""Pins the oracle: the C restatement against the golden fixtures (made by the
reference itself) and, where the compiled reference is present, against the
reference directly on fresh seeded inputs.  CPU only."""
import os
import tempfile

import numpy as np
import pytest

import oracle
from pawan_b200 import geometry as g
from pawan_b200 import state_to_union, union_to_state
from helpers import load, rms_rel, max_rel, split_rates

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("name", ["ring64_solve", "pair64_solve", "helix3_solve"])
def test_restatement_matches_golden_solve(name):
    d = load(name)
    u_ref, da_ref = split_rates(d["counts"], d["rates"])
    u, da = oracle.pairs(d["pos"], d["vor"], d["rad"], d["vol"], float(d["nu"]))
    assert rms_rel(u, u_ref) < 1e-13
    assert rms_rel(da, da_ref) < 1e-13
    assert max_rel(u, u_ref) < 1e-12 and max_rel(da, da_ref) < 1e-12


@pytest.mark.parametrize("name", ["ring64_rk4", "pair64_rk4"])
def test_restatement_matches_golden_rk4(name):
    d = load(name)
    p, v = oracle.rk4_step(d["pos"], d["vor"], d["rad"], d["vol"], float(d["nu"]), float(d["dt"]),
                           int(d["nsteps"]))
    out = union_to_state(list(d["counts"]), p, v)
    assert rms_rel(out, d["final_state"]) < 1e-14
    # the increments themselves, not just the states
    assert rms_rel(out - d["state"], d["final_state"] - d["state"]) < 1e-11


def test_restatement_matches_golden_diagnostics():
    d = load("pair64_diag")
    O, I, A = oracle.linear_diagnostics(d["pos"], d["vor"])
    scale = np.abs(d["vor"]).sum()
    assert np.abs(O - d["total_vorticity"]).max() < 1e-14 * scale
    # sums of many terms that largely cancel: compare against the term scale
    r2a = (np.linalg.norm(d["pos"], axis=1) ** 2 * np.linalg.norm(d["vor"], axis=1)).sum()
    assert np.abs(I - d["linear_impulse"]).max() < 1e-14 * r2a
    assert np.abs(A - d["angular_impulse"]).max() < 1e-14 * r2a
    assert abs(oracle.enstrophy(d["pos"], d["vor"], d["rad"]) / d["enstrophy"] - 1) < 1e-12
    h = oracle.helicity(d["pos"], d["vor"], d["rad"])
    assert abs(h - d["helicity"]) < 1e-10 * abs(d["enstrophy"])
    wid = np.repeat(np.arange(len(d["counts"])), d["counts"])
    assert abs(oracle.kinetic_energy(wid, d["pos"], d["vor"], d["rad"]) / d["kinetic_energy"] - 1) < 1e-12


def test_golden_wake_file_layout():
    """The .wake frames of __integration::integrate: t, nWake, then per wake N,
    x (N x 3), alpha (N x 3), s (N)."""
    d = load("ring16_integrate")
    raw = d["wake_bytes"].tobytes()
    n = int(d["counts"].sum())
    frame = 8 + 8 + 8 + 8 * (7 * n)
    assert len(raw) == frame * (int(d["nsteps"]) + 1)
    t0 = np.frombuffer(raw[:8], dtype=np.float64)[0]
    assert t0 == 0.0
    nw = np.frombuffer(raw[8:16], dtype=np.uint64)[0]
    assert nw == 1
    x0 = np.frombuffer(raw[24:24 + 24 * n], dtype=np.float64).reshape(n, 3)
    assert np.array_equal(x0, d["pos"])
    t_last = np.frombuffer(raw[frame * 2: frame * 2 + 8], dtype=np.float64)[0]
    assert t_last == pytest.approx(0.02)


@needs_ref
@pytest.mark.parametrize("parallel", [False, True])
def test_restatement_matches_reference_fresh_inputs(parallel):
    sc = g.ring_pair(n_stations=12, seed=101, nu=5e-4)
    pos, vor, rad, vol = sc.union()
    ref = oracle.RefSystem(sc.counts, pos, vor, rad, vol, sc.nu, parallel=parallel)
    ref.solve()
    u_ref, da_ref = ref.union_rates()
    u, da = oracle.pairs(pos, vor, rad, vol, sc.nu)
    assert rms_rel(u, u_ref) < 1e-13 and rms_rel(da, da_ref) < 1e-13


@needs_ref
def test_reference_rates_layout_and_wake_rates_agree():
    sc = g.ring_pair(n_stations=3, seed=5, nu=1e-3)
    ref = oracle.RefSystem(sc.counts, *sc.union(), sc.nu)
    ref.solve()
    u, da = split_rates(sc.counts, ref.get_rates())
    u2, da2 = ref.union_rates()
    assert np.array_equal(u, u2) and np.array_equal(da, da2)


@needs_ref
def test_restatement_sampled_targets_match_full():
    sc = g.single_ring(n_stations=16, seed=3, nu=1e-3)
    pos, vor, rad, vol = sc.union()
    u, da = oracle.pairs(pos, vor, rad, vol, sc.nu)
    t = np.array([0, 5, 77, 127])
    ut, dat = oracle.pairs(pos, vor, rad, vol, sc.nu, targets=t)
    assert np.array_equal(ut, u[t]) and np.array_equal(dat, da[t])


@needs_ref
def test_reference_state_roundtrip():
    sc = g.helical_wake(n_stations=2, seed=9, filaments=2, turns=1.0)
    ref = oracle.RefSystem(sc.counts, *sc.union(), sc.nu)
    st = sc.state()
    assert np.array_equal(ref.get_states(), st)
    p, v = state_to_union(sc.counts, st)
    assert np.array_equal(union_to_state(sc.counts, p, v), st)


def test_conservation_of_total_vorticity_rate():
    """Each reference pair adds +da to the target and -da to the source
    (interaction_utils.h:471-475), so the rates sum to zero."""
    d = load("pair64_solve")
    _, da = split_rates(d["counts"], d["rates"])
    assert np.abs(da.sum(axis=0)).max() < 1e-12 * np.abs(da).sum()


@pytest.mark.parametrize("name", ["pair64_influence", "vring1_influence"])
def test_restatement_matches_golden_influence(name):
    """The vorticity field of __interaction::influence (interaction.cpp:110-155)."""
    d = load(name)
    k = oracle.influence(d["pos"], d["vor"], d["rad"])
    assert rms_rel(k, d["field"]) < 1e-13 and max_rel(k, d["field"]) < 1e-12


@needs_ref
def test_restatement_influence_matches_reference_fresh_inputs():
    sc = g.helical_wake(n_stations=3, seed=17, filaments=3, turns=1.0)
    pos, vor, rad, vol = sc.union()
    rad = rad * np.random.default_rng(3).uniform(0.8, 1.2, rad.shape)  # mixed radii
    ref = oracle.RefSystem(sc.counts, pos, vor, rad, vol, 0.0)
    k_ref = ref.influence()
    k = oracle.influence(pos, vor, rad)
    assert rms_rel(k, k_ref) < 1e-13 and max_rel(k, k_ref) < 1e-12


@needs_ref
def test_reference_vring_resolve_reproduces_golden():
    """__resolve::rebuild on the reference's __vring (influence matrix by unit
    strengths, LU solve against the ideal Gaussian core field) through the GSL
    shim's LU routines."""
    d = load("vring1_resolve")
    v = oracle.RefVring(float(d["radius"]), float(d["core"]), int(d["layers"]))
    pos, _, rad, vol = v.particles()
    assert np.array_equal(pos, d["pos"]) and np.array_equal(rad, d["rad"])
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        os.chdir(tmp)
        try:
            s = v.resolve()
        finally:
            os.chdir(cwd)
    v.close()
    assert np.array_equal(s, d["strengths"])


def test_restatement_matches_golden_gaussian_kernel():
    """The reference compiled with its Gaussian kernel (gaussian.h): rates, two
    RK4 steps, helicity (enstrophy is the reference's stub 0) and the field."""
    d = load("pair64_gauss")
    args = (d["pos"], d["vor"], d["rad"], d["vol"])
    u_ref, da_ref = split_rates(d["counts"], d["rates"])
    u, da = oracle.pairs(*args, float(d["nu"]), kernel="gaussian")
    assert rms_rel(u, u_ref) < 1e-13 and rms_rel(da, da_ref) < 1e-13
    p, v = oracle.rk4_step(*args, float(d["nu"]), float(d["dt"]), int(d["nsteps"]), kernel="gaussian")
    out = union_to_state(list(d["counts"]), p, v)
    assert rms_rel(out - d["state"], d["final_state"] - d["state"]) < 1e-11
    assert float(d["enstrophy"]) == 0.0
    assert oracle.enstrophy(d["pos"], d["vor"], d["rad"], kernel="gaussian") == 0.0
    h = oracle.helicity(d["pos"], d["vor"], d["rad"], kernel="gaussian")
    assert abs(h - d["helicity"]) <= 1e-11 * abs(d["helicity"]) + 1e-18
    k = oracle.influence(d["pos"], d["vor"], d["rad"], kernel="gaussian")
    assert rms_rel(k, d["field"]) < 1e-13


@needs_ref
def test_gaussian_reference_differs_from_default_kernel():
    """The two compiled references really run different kernels."""
    sc = g.ring_pair(n_stations=6, seed=19, nu=1e-3)
    pos, vor, rad, vol = sc.union()
    a = oracle.RefSystem(sc.counts, pos, vor, rad, vol, sc.nu)
    b = oracle.RefSystem(sc.counts, pos, vor, rad, vol, sc.nu, kernel="gaussian")
    a.solve()
    b.solve()
    assert rms_rel(a.get_rates(), b.get_rates()) > 1e-3
