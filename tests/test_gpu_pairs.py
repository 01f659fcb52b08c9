"""Parity of the CUDA all-pairs interaction with the reference, through the C ABI.

Tolerances (tests/helpers.py): FP32 pair math with FP64 accumulation -- RMS
relative error <= 1e-5 and max error <= 1e-4 of the max reference value, for
velocity and vorticity rate separately; plain FP64 -- RMS <= 1e-12, max <= 1e-11;
tuned FP64 -- RMS <= 1e-10, max <= 1e-9.
"""
import numpy as np
import pytest

import oracle
import pawan_b200
from pawan_b200 import System
from pawan_b200 import union_to_state as union_state
from pawan_b200 import geometry as g
from helpers import load, max_rel, rms_rel, split_rates, tol

pytestmark = pytest.mark.gpu

PRECS = ["f32", "f64", "f64_plain"]


def check(prec, u, da, u_ref, da_ref):
    t_rms, t_max = tol(prec)
    assert rms_rel(u, u_ref) <= t_rms, ("u rms", rms_rel(u, u_ref))
    assert rms_rel(da, da_ref) <= t_rms, ("da rms", rms_rel(da, da_ref))
    assert max_rel(u, u_ref) <= t_max, ("u max", max_rel(u, u_ref))
    assert max_rel(da, da_ref) <= t_max, ("da max", max_rel(da, da_ref))


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", ["ring64_solve", "pair64_solve", "helix3_solve"])
def test_solve_matches_reference_golden(ctx, name, prec):
    d = load(name)
    counts = [int(c) for c in d["counts"]]
    s = System(ctx, counts, float(d["nu"]), prec)
    s.set_particles(d["pos"], d["vor"], d["rad"], d["vol"])
    s.solve()
    rates = s.get_rates()
    u, da = split_rates(counts, rates)
    u_ref, da_ref = split_rates(counts, d["rates"])
    check(prec, u, da, u_ref, da_ref)
    # per-wake accessor agrees with the rate vector
    uu, dd = s.union_rates()
    assert np.array_equal(uu, u) and np.array_equal(dd, da)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("prec", PRECS)
def test_solve_matches_reference_fresh(ctx, prec):
    sc = g.ring_pair(n_stations=40, seed=202, nu=7e-4)  # N = 640, two wakes
    pos, vor, rad, vol = sc.union()
    ref = oracle.RefSystem(sc.counts, pos, vor, rad, vol, sc.nu)
    ref.solve()
    s = System.from_scenario(ctx, sc, prec)
    s.solve()
    check(prec, *s.union_rates(), *ref.union_rates())
    assert np.array_equal(s.get_rates(), s.get_rates())


@pytest.mark.parametrize("n", [2, 3, 31, 127, 128, 129, 255, 257, 1000, 4099])
def test_ragged_sizes_against_restatement(ctx, n):
    rng = np.random.default_rng(n)
    pos = rng.uniform(-1, 1, (n, 3))
    vor = rng.normal(0, 0.01, (n, 3))
    rad = rng.uniform(0.05, 0.2, n)
    vol = rng.uniform(1e-4, 2e-4, n)
    u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, 1e-3)
    for prec in PRECS:
        s = System(ctx, [n], 1e-3, prec)
        s.set_particles(pos, vor, rad, vol)
        s.solve()
        check(prec, *s.union_rates(), u_ref, da_ref)
    # FP32 through both near passes (random radii: the general scalars; ragged
    # last tiles: sources past the end staged as far, zero-strength particles)
    s = System(ctx, [n], 1e-3, "f32")
    s.set_particles(pos, vor, rad, vol)
    for tb in (128, 256):
        for split in (1, 2):
            s.set_config(threads=tb, unroll=4, packed=1, split_near=split)
            s.solve()
            check("f32", *s.union_rates(), u_ref, da_ref)


@pytest.mark.parametrize("prec", PRECS)
def test_coincident_particles_give_nan_where_the_reference_does(ctx, prec):
    """Distinct particles at one position: the reference's kernel is singular
    at rho = 0 (q and F divide by rho, highorder.h:58-59), so in its solve
    those particles' rates are NaN and every other particle's are finite.
    The GPU paths exclude only the self pair, by index, as the reference does
    (interaction.cpp:158-173): NaN in the same rows, the other rows within
    tolerance.  One coincident pair shares a 128-tile, one spans two tiles."""
    rng = np.random.default_rng(11)
    n = 300
    pos = rng.uniform(-1, 1, (n, 3))
    pos[100] = pos[7]
    pos[250] = pos[40]
    vor = rng.normal(0, 0.01, (n, 3))
    rad = rng.uniform(0.05, 0.2, n)
    vol = rng.uniform(1e-4, 2e-4, n)
    if oracle.ref_available():
        r = oracle.RefSystem([n], pos, vor, rad, vol, 1e-3)
        r.solve()
        u_ref, da_ref = r.union_rates()
    else:
        u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, 1e-3)
    bad = np.isnan(u_ref).any(axis=1) | np.isnan(da_ref).any(axis=1)
    assert sorted(np.flatnonzero(bad)) == [7, 40, 100, 250]
    s = System(ctx, [n], 1e-3, prec)
    s.set_particles(pos, vor, rad, vol)
    # FP32: the default tiling, then the scalar and the packed near pass
    configs = [None] + ([dict(threads=128, unroll=4, packed=2, split_near=sp) for sp in (1, 2)]
                        if prec == "f32" else [])
    for cfg in configs:
        if cfg:
            s.set_config(**cfg)
        s.solve()
        u, da = s.union_rates()
        assert np.array_equal(np.isnan(u).all(axis=1) & np.isnan(da).all(axis=1), bad), cfg
        assert np.isfinite(u[~bad]).all() and np.isfinite(da[~bad]).all(), cfg
        check(prec, u[~bad], da[~bad], u_ref[~bad], da_ref[~bad])


def test_many_wakes_union(ctx):
    """Five wakes of uneven size: all pairs over the union, like interact()."""
    rng = np.random.default_rng(5)
    counts = [17, 200, 1, 64, 333]
    n = sum(counts)
    pos = rng.uniform(-1, 1, (n, 3))
    vor = rng.normal(0, 0.01, (n, 3))
    rad = rng.uniform(0.05, 0.2, n)
    vol = rng.uniform(1e-4, 2e-4, n)
    u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, 2e-3)
    s = System(ctx, counts, 2e-3, "f32")
    s.set_particles(pos, vor, rad, vol)
    s.solve()
    check("f32", *s.union_rates(), u_ref, da_ref)


# (threads, threads per target, targets per thread, unroll, blocks per SM) as compiled
F32_TILINGS = [(128, 1, 1, 2, 0), (128, 1, 1, 4, 0), (128, 2, 1, 2, 0), (128, 2, 1, 4, 0),
               (128, 4, 1, 4, 0), (128, 1, 2, 1, 0), (128, 1, 2, 2, 0), (128, 1, 1, 2, 5),
               (128, 1, 1, 4, 5), (128, 1, 1, 2, 6), (128, 1, 1, 4, 6), (256, 1, 1, 2, 0),
               (256, 1, 1, 4, 0), (256, 2, 1, 4, 0), (256, 4, 1, 4, 0), (256, 1, 2, 1, 0),
               (256, 1, 2, 2, 0), (256, 1, 1, 4, 3)]
# packed far path (two sources per FP32x2 instruction): (threads, unroll, blocks per SM,
# mode: 1 = 1/rho^2 from the MUFU reciprocal, 2 = from rsqrt squared)
F32_PACKED = [(128, 1, 0, 1), (128, 2, 0, 1), (128, 4, 0, 1), (128, 1, 5, 1), (128, 2, 5, 1),
              (128, 2, 0, 2), (128, 4, 0, 2), (256, 2, 0, 1), (256, 4, 0, 1), (256, 2, 0, 2),
              (256, 4, 0, 2)]


@pytest.mark.parametrize("tb,unroll,minb,mode", F32_PACKED)
def test_every_packed_f32_tiling(ctx, tb, unroll, minb, mode):
    sc = g.ring_pair(n_stations=70, seed=34, nu=1e-3)
    pos, vor, rad, vol = sc.union()
    s = System.from_scenario(ctx, sc, "f32")
    for nu in (1e-3, 0.0):
        s.set_nu(nu)
        u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, nu)
        for ips in (1, 16, 64):
            s.set_config(tb, 1, unroll, ips, blocks_per_sm=minb, packed=mode)
            s.solve()
            check("f32", *s.union_rates(), u_ref, da_ref)
        if unroll == 4 and minb == 0:
            # the same with the near tile pairs in a pass of their own, scalar and packed
            for split in (1, 2):
                s.set_config(tb, 1, unroll, 16, packed=mode, split_near=split)
                s.solve()
                check("f32", *s.union_rates(), u_ref, da_ref)


@pytest.mark.parametrize("tb,p,r,unroll,minb", F32_TILINGS)
def test_every_f32_tiling(ctx, tb, p, r, unroll, minb):
    sc = g.ring_pair(n_stations=70, seed=33, nu=1e-3)  # N = 1120: ragged tiles
    pos, vor, rad, vol = sc.union()
    u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, sc.nu)
    s = System.from_scenario(ctx, sc, "f32")
    for ips in (1, 16, 64):
        s.set_config(tb, p, unroll, ips, targets_per_thread=r, blocks_per_sm=minb)
        s.solve()
        check("f32", *s.union_rates(), u_ref, da_ref)
    s.set_nu(0.0)
    s.solve()
    check("f32", *s.union_rates(), *oracle.pairs(pos, vor, rad, vol, 0.0))


def _separated_rings(alternate: bool):
    """Three rings far apart (most tile pairs take the far formulation), the
    second with a larger smoothing radius; with `alternate` the third ring's
    particles alternate between two radii (no uniform-radius tile pairs)."""
    rng = np.random.default_rng(77)
    wakes = [g.ring(1.0, 0.1, 1.0, 48, 0.0, rng), g.ring(0.8, 0.1, -0.7, 40, 3.0, rng),
             g.ring(1.2, 0.08, 1.3, 56, -2.5, rng)]
    wakes[1].rad *= 1.3
    if alternate:
        wakes[2].rad[1::2] *= 0.7
    counts = [w.n for w in wakes]
    pos = np.concatenate([w.pos for w in wakes])
    vor = np.concatenate([w.vor for w in wakes])
    rad = np.concatenate([w.rad for w in wakes])
    vol = np.concatenate([w.vol for w in wakes])
    return counts, pos, vor, rad, vol


@pytest.mark.parametrize("alternate", [False, True])
def test_far_formulations_every_tiling(ctx, alternate):
    """Uniform-radius and mixed-radius far tiles, scalar and packed paths."""
    counts, pos, vor, rad, vol = _separated_rings(alternate)
    s = System(ctx, counts, 1e-3, "f32")
    s.set_particles(pos, vor, rad, vol)
    for nu in (1e-3, 0.0):
        s.set_nu(nu)
        u_ref, da_ref = oracle.pairs(pos, vor, rad, vol, nu)
        for tb, p, r, unroll, minb in F32_TILINGS:
            s.set_config(tb, p, unroll, 16, targets_per_thread=r, blocks_per_sm=minb)
            s.solve()
            check("f32", *s.union_rates(), u_ref, da_ref)
        for tb, unroll, minb, mode in F32_PACKED:
            s.set_config(tb, 1, unroll, 16, blocks_per_sm=minb, packed=mode)
            s.solve()
            check("f32", *s.union_rates(), u_ref, da_ref)


def test_nu_zero_matches_and_set_nu(ctx):
    sc = g.single_ring(n_stations=50, seed=8, nu=0.0)
    pos, vor, rad, vol = sc.union()
    s = System.from_scenario(ctx, sc, "f32")
    s.solve()
    check("f32", *s.union_rates(), *oracle.pairs(pos, vor, rad, vol, 0.0))
    s.set_nu(5e-3)
    s.solve()
    check("f32", *s.union_rates(), *oracle.pairs(pos, vor, rad, vol, 5e-3))


def test_deterministic_bits(ctx):
    sc = g.ring_pair(n_stations=300, seed=9, nu=1e-4)
    s = System.from_scenario(ctx, sc, "f32")
    s.solve()
    a = s.get_rates()
    for _ in range(3):
        s.solve()
        assert np.array_equal(s.get_rates(), a)


def test_total_vorticity_rate_conserved(ctx):
    """Pair terms are antisymmetric, so sum dalpha = 0 up to rounding."""
    sc = g.ring_pair(n_stations=256, seed=10, nu=1e-3)
    s = System.from_scenario(ctx, sc, "f32")
    s.solve()
    _, da = s.union_rates()
    assert np.abs(da.sum(axis=0)).max() < 1e-5 * np.abs(da).sum()


def test_state_roundtrip_exact(ctx):
    sc = g.helical_wake(n_stations=12, seed=4, filaments=3, turns=1.0)
    s = System.from_scenario(ctx, sc, "f32")
    st = sc.state()
    assert np.array_equal(s.get_states(), st)
    st2 = st + 1e-3
    s.set_states(st2)
    assert np.array_equal(s.get_states(), st2)


def test_invalid_arguments_raise(ctx):
    with pytest.raises(pawan_b200.PawanError):
        System(ctx, [], 0.0)
    with pytest.raises(pawan_b200.PawanError):
        System(ctx, [1], 0.0)  # a single particle interacts with nothing
    with pytest.raises(pawan_b200.PawanError):
        System(ctx, [5, 0, 7], 0.0)  # an empty wake (the reference's GSL aborts on it)
    with pytest.raises(pawan_b200.PawanError):
        System(ctx, [10], -1.0)
    s = System(ctx, [10], 0.0)
    with pytest.raises(pawan_b200.PawanError):
        s.solve()  # no particles yet
    with pytest.raises(pawan_b200.PawanError):
        s.set_config(96, 1, 2, 16)


# The tilings the autotuner times (pawan_tile_candidates; tests/test_abi.py
# checks this list against the library's): (threads, threads per target,
# targets per thread, unroll, blocks per SM, packed mode).
TUNE_CANDIDATES = [(tb,) + sh + (0,) for tb in (128, 256) for sh in (
    (1, 1, 4, 0, 0), (2, 1, 4, 0, 0), (4, 1, 4, 0, 0), (1, 2, 1, 0, 0), (1, 2, 2, 0, 0),
    (1, 1, 4, 5, 0), (1, 1, 1, 0, 1), (1, 1, 2, 0, 1), (1, 1, 4, 0, 1), (1, 1, 2, 5, 1),
    (1, 1, 2, 0, 2), (1, 1, 4, 0, 2))
    if not (tb == 256 and sh in ((1, 1, 4, 5, 0), (1, 1, 1, 0, 1), (1, 1, 2, 5, 1)))]
# ... and with a separate near pass (the last field: 1 scalar, 2 packed)
TUNE_CANDIDATES += [(tb, 1, 1, 4, 0, pk, sp) for sp in (1, 2) for tb in (128, 256) for pk in (1, 2)]
# the tiling the default bench run's autotuner picks on the ring pair, and the
# library's default tiling
TIMED_TILING = (256, 1, 1, 4, 0, 2, 0)
DEFAULT_TILING = (128, 1, 1, 4, 0, 2, 0)
FULL_SAMPLES = 4096


@pytest.fixture(scope="module")
def full(ctx):
    """Per workload, made on first use: (system, sampled targets, oracle rates
    at them), the oracle summing 4,096 targets over all N sources in FP64."""
    made = {}

    def get(name):
        if name not in made:
            sc = g.ring_pair(steps=1) if name == "ring_pair" else g.helical_wake(steps=1)
            pos, vor, rad, vol = sc.union()
            t = np.sort(np.random.default_rng(0).choice(sc.n, FULL_SAMPLES, replace=False))
            made[name] = (System.from_scenario(ctx, sc, "f32"), t,
                          oracle.pairs(pos, vor, rad, vol, sc.nu, targets=t))
        return made[name]
    yield get
    for s, _, _ in made.values():
        s.close()


def _check_full(full, name, tiling, ips):
    s, t, (u_ref, da_ref) = full(name)
    tb, p, r, unroll, minb, mode, split = tiling
    s.set_config(tb, p, unroll, ips, targets_per_thread=r, blocks_per_sm=minb, packed=mode,
                 split_near=split)
    s.solve()
    u, da = s.union_rates()
    check("f32", u[t], da[t], u_ref, da_ref)
    assert np.abs(da.sum(axis=0)).max() < 1e-5 * np.abs(da).sum()


@pytest.mark.parametrize("tiling", TUNE_CANDIDATES, ids=lambda c: "tiling" + "-".join(map(str, c)))
@pytest.mark.parametrize("name", ["ring_pair", "helical_wake"])
def test_full_size_every_candidate_tiling(full, name, tiling):
    """N = 131,072 (ring pair) and 262,144 (helical wake) in FP32 with every
    tiling the autotuner can pick, at its finest chunking (128 work items per
    resident block): 4,096 sampled targets against the FP64 restatement
    summed over all N sources."""
    _check_full(full, name, tiling, 128)


@pytest.mark.parametrize("ips", [4, 8, 16, 32, 64])
@pytest.mark.parametrize("tiling", [TIMED_TILING, DEFAULT_TILING], ids=["timed", "default"])
@pytest.mark.parametrize("name", ["ring_pair", "helical_wake"])
def test_full_size_timed_tiling_every_chunking(full, name, tiling, ips):
    """The bench's autotuned tiling (256 threads, packed mode 2) and the
    library default (128 threads, mode 2) at every chunking the autotuner
    times, at full size against the FP64 restatement."""
    _check_full(full, name, tiling, ips)


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("gap", [3.0, 4.5, 5.5, 6.5, 10.0, 15.0, 17.0, 20.0])
def test_tile_classes_at_their_boundaries(ctx, gap, mixed):
    """Two compact clusters of 256 particles (two 128-tiles each) whose boxes
    are `gap` smoothing radii apart: near (< 4 s), far with the Z terms
    (4 s .. 6 s), far without them (>= 6 s, where Z is below 3e-9 of q) and
    far without them by the two-term series of the smoothing factor (>= 16 s,
    truncation below 3e-8).
    The whole solve against the FP64 oracle; then the cross-cluster part at
    cluster A on its own, by linearity: the same system solved with cluster
    B's strengths doubled, minus the first solve, is at A exactly the part of
    A's rates that B's strengths drive (A's own tiles compute identically in
    both solves), compared with the same difference in the oracle.  nu != 0;
    packed and scalar tilings; one smoothing radius (the uniform-radius
    forms) or radii in [0.8 s, 1.2 s] (the general forms; the Z-free class
    then starts at 7.2 s and the series at 19.2 s)."""
    rng = np.random.default_rng(int(gap * 10))
    s = 0.05
    n = 256
    a = rng.uniform(-0.5 * s, 0.5 * s, (n, 3))
    b = rng.uniform(-0.5 * s, 0.5 * s, (n, 3))
    b[:, 0] += (gap + 1.0) * s  # box gap = gap * s
    pos = np.concatenate([a, b])
    vor = rng.normal(size=(2 * n, 3)) * 1e-3
    tol = 1e-5
    if gap >= 15.0:
        # from about 15 s on, the stretching that random strengths of a
        # distant cluster drive cancels to a small fraction of its terms (the
        # FP64-vs-FP32 distance of the exact Z-free form reaches 1.3e-5 at
        # 17 s); a common strength direction keeps it well conditioned, so a
        # tighter bound applies
        vor[n:] += np.array([1e-3, 2e-3, -1.5e-3])
        tol = 2e-6
    vor2 = vor.copy()
    vor2[n:] *= 2.0
    rad = s * rng.uniform(0.8, 1.2, 2 * n) if mixed else np.full(2 * n, s)
    vol = np.full(2 * n, 1e-5)
    nu = 1e-3
    u1, da1 = oracle.pairs(pos, vor, rad, vol, nu)
    u2, da2 = oracle.pairs(pos, vor2, rad, vol, nu)
    du_ref, dda_ref = (u2 - u1)[:n], (da2 - da1)[:n]
    st1, st2 = union_state([2 * n], pos, vor), union_state([2 * n], pos, vor2)
    sysm = System(ctx, [2 * n], nu, "f32")
    sysm.set_particles(pos, vor, rad, vol)
    configs = [dict(threads=tb, threads_per_target=1, unroll=unroll, items_per_slot=16,
                    blocks_per_sm=minb, packed=mode) for tb, unroll, minb, mode in F32_PACKED[:4]]
    configs += [dict(threads=tb, threads_per_target=p, unroll=unroll, items_per_slot=16,
                     targets_per_thread=r, blocks_per_sm=minb) for tb, p, r, unroll, minb in F32_TILINGS[:6]]
    # the separate near pass, scalar and packed
    configs += [dict(threads=128, unroll=4, items_per_slot=16, packed=mode, split_near=sp)
                for sp in (1, 2) for mode in (1, 2)]
    for cfg in configs:
        sysm.set_config(**cfg)
        sysm.set_states(st1)
        sysm.solve()
        ug1, dag1 = sysm.union_rates()
        check("f32", ug1, dag1, u1, da1)
        sysm.set_states(st2)
        sysm.solve()
        ug2, dag2 = sysm.union_rates()
        du, dda = (ug2 - ug1)[:n], (dag2 - dag1)[:n]
        assert rms_rel(du, du_ref) < tol and rms_rel(dda, dda_ref) < tol, \
            (cfg, rms_rel(du, du_ref), rms_rel(dda, dda_ref))


@pytest.mark.parametrize("tiling", [TIMED_TILING, DEFAULT_TILING, (128, 2, 1, 4, 0, 0, 0), (128, 1, 2, 2, 0, 0, 0),
                                    (256, 1, 1, 4, 0, 1, 1), (256, 1, 1, 4, 0, 2, 2), (128, 1, 1, 4, 0, 1, 2)],
                         ids=["timed", "default", "two-threads-per-target", "two-targets-per-thread",
                              "near-pass", "packed-near-pass", "packed-near-pass-128"])
def test_chunk_sums_inside_the_launch(ctx, tiling):
    """The pair kernels sum a target tile's chunk partials inside the launch
    (the block completing the tile, in chunk order).  With the tiling fixed,
    the chunking changes only how the FP64 sums are grouped -- every FP32
    tile sum is the same -- so plans of 1 to 1,024 work items per resident
    block (from a few source chunks per target tile to one per source tile)
    agree to FP64 rounding; a chunk lost or counted twice would differ by
    percents.  Also across repeated launches (the tile counters re-arm) and a
    ragged last tile.  (A single chunk, where items write the rates directly,
    is the small systems of test_ragged_sizes_against_restatement.)"""
    sc = g.ring_pair(n_stations=300, seed=61, nu=1e-4)  # N = 4,800: ragged target tiles
    tb, p, r, unroll, minb, mode, split = tiling
    s = System.from_scenario(ctx, sc, "f32")
    results = []
    for ips in (1, 2, 8, 32, 128, 1024):
        s.set_config(tb, p, unroll, ips, targets_per_thread=r, blocks_per_sm=minb, packed=mode,
                     split_near=split)
        s.solve()
        first = s.union_rates()
        s.solve()
        again = s.union_rates()
        assert np.array_equal(first[0], again[0]) and np.array_equal(first[1], again[1])
        results.append(first)
    u0, d0 = results[0]
    for u, d in results[1:]:
        assert rms_rel(u, u0) < 1e-13 and rms_rel(d, d0) < 1e-13, (rms_rel(u, u0), rms_rel(d, d0))
    s.close()
