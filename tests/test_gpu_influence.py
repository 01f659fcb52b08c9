"""The vorticity field (the reference's __interaction::resolve -> influence,
src/interaction/interaction.cpp:45-47, 110-155) on the GPU, and the reference's
own influence-matrix resolve (src/resolve/resolve.cpp:10-57) driven through
the drop-in class.  FP64 throughout: tolerance TOL_F64 (RMS 1e-12, max 1e-11)."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

import oracle
from pawan_b200 import System
from pawan_b200 import geometry as g
from helpers import TOL_F64_MAX, TOL_F64_RMS, load, max_rel, rms_rel

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libpawan_dropin.so")
needs_lib = pytest.mark.skipif(not os.path.exists(LIB), reason="drop-in harness not built")
_dp = ctypes.POINTER(ctypes.c_double)
_szp = ctypes.POINTER(ctypes.c_size_t)


def check(k, k_ref):
    assert rms_rel(k, k_ref) <= TOL_F64_RMS, rms_rel(k, k_ref)
    assert max_rel(k, k_ref) <= TOL_F64_MAX, max_rel(k, k_ref)


@pytest.mark.parametrize("name", ["pair64_influence", "vring1_influence"])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_influence_matches_golden(ctx, name, prec):
    d = load(name)
    s = System(ctx, [int(c) for c in d["counts"]], 0.0, prec)
    s.set_particles(d["pos"], d["vor"], d["rad"], d["vol"])
    check(s.influence(), d["field"])


def test_influence_matches_oracle_mixed_radii_many_wakes(ctx):
    sc = g.helical_wake(n_stations=96, seed=23, filaments=4, turns=2.0)  # N = 3,072
    pos, vor, rad, vol = sc.union()
    rad = rad * np.random.default_rng(5).uniform(0.7, 1.3, rad.shape)
    s = System(ctx, sc.counts, 0.0, "f32")
    s.set_particles(pos, vor, rad, vol)
    check(s.influence(), oracle.influence(pos, vor, rad))


@pytest.mark.parametrize("kernel", ["highorder", "gaussian"])
def test_influence_columns_bit_identical_to_single_column(ctx, kernel):
    """Eleven strength columns (one full group of eight and a partial one) in
    one call: each column equals the single-column field of that strength bit
    for bit, matches the oracle, and the system's own strengths are untouched."""
    sc = g.ring_pair(n_stations=40, seed=31, nu=0.0)  # N = 640, not a multiple of 128
    pos, vor, rad, vol = sc.union()
    rad = rad * np.random.default_rng(6).uniform(0.8, 1.2, rad.shape)
    s = System(ctx, sc.counts, 0.0, "f32")
    s.set_kernel(kernel)
    s.set_particles(pos, vor, rad, vol)
    own = s.influence()
    cols = np.random.default_rng(7).standard_normal((11, sc.n, 3))
    k = s.influence_columns(cols)
    assert np.array_equal(s.influence(), own)
    for c in range(cols.shape[0]):
        s.set_particles(pos, cols[c], rad, vol)
        assert np.array_equal(k[c], s.influence()), c
        check(k[c], oracle.influence(pos, cols[c], rad, kernel=kernel))


def test_influence_columns_split_over_launches(ctx):
    """More columns than the 256 MiB device scratch holds (1,365 columns of
    N = 4,096): the columns run in two launches, and the columns on either
    side of the split, and the last, equal single-column solves."""
    rng = np.random.default_rng(8)
    n = 4096
    pos = rng.uniform(-1, 1, (n, 3))
    rad = rng.uniform(0.05, 0.1, n)
    vol = np.full(n, 1e-4)
    ncols = 1400
    fit = (256 << 20) // (2 * 3 * n * 8)
    assert fit < ncols
    cols = rng.standard_normal((ncols, n, 3))
    s = System(ctx, [n], 0.0, "f32")
    s.set_particles(pos, cols[0], rad, vol)
    k = s.influence_columns(cols)
    for c in (0, fit - 1, fit, ncols - 1):
        s.set_particles(pos, cols[c], rad, vol)
        assert np.array_equal(k[c], s.influence()), c


def test_influence_columns_rejects_bad_sizes(ctx):
    sc = g.single_ring(n_stations=8, seed=1)
    s = System.from_scenario(ctx, sc, "f32")
    a = np.zeros((2, sc.n, 3))
    k = np.empty_like(a)
    f = s._lib.pawan_system_influence_columns
    assert f(s.handle, 2, a.ctypes.data_as(_dp), k.ctypes.data_as(_dp), a.size - 3) == 1
    assert f(s.handle, 0, a.ctypes.data_as(_dp), k.ctypes.data_as(_dp), 0) == 1
    assert f(s.handle, 2, None, k.ctypes.data_as(_dp), a.size) == 1
    with pytest.raises(ValueError):
        s.influence_columns(np.zeros((2, sc.n + 1, 3)))


def test_influence_follows_the_state(ctx):
    """After RK4 steps and after set_states the field is that of the new state."""
    sc = g.ring_pair(n_stations=64, seed=24, nu=1e-3)
    pos, vor, rad, vol = sc.union()
    s = System.from_scenario(ctx, sc, "f64")
    s.rk4(sc.dt, 2)
    from pawan_b200 import state_to_union
    p1, v1 = state_to_union(sc.counts, s.get_states())
    check(s.influence(), oracle.influence(p1, v1, rad))
    s.set_states(sc.state())
    check(s.influence(), oracle.influence(pos, vor, rad))


def test_influence_rejects_bad_sizes(ctx):
    sc = g.single_ring(n_stations=8, seed=1)
    s = System.from_scenario(ctx, sc, "f32")
    bad = np.empty(3 * sc.n - 1)
    st = s._lib.pawan_system_influence(s.handle, bad.ctypes.data_as(_dp), bad.size)
    assert st == 1  # PAWAN_ERR_INVALID


@pytest.fixture(scope="module")
def lib():
    L = ctypes.CDLL(LIB)
    L.dropin_influence.argtypes = [ctypes.c_int, _szp, _dp, _dp, _dp, _dp, _dp, _dp]
    L.dropin_vring_resolve.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp, _dp]
    L.dropin_vring_resolve_batched.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp,
                                               _dp, ctypes.POINTER(ctypes.c_int)]
    return L


@needs_lib
def test_dropin_resolve_hook_matches_reference(lib):
    """__cuda::influence (behind resolve()) against the reference __interaction."""
    sc = g.ring_pair(n_stations=24, seed=25, nu=0.0)
    pos, vor, rad, vol = (np.ascontiguousarray(a) for a in sc.union())
    cnt = np.asarray(sc.counts, dtype=np.uintp)
    gpu, cpu = np.empty((sc.n, 3)), np.empty((sc.n, 3))
    assert lib.dropin_influence(len(sc.counts), cnt.ctypes.data_as(_szp),
                                *[a.ctypes.data_as(_dp) for a in (pos, vor, rad, vol, gpu, cpu)]) == 0
    check(gpu, cpu)


@needs_lib
def test_dropin_vring_resolve_matches_reference(lib):
    """The reference's __resolve::rebuild over a __vring: 9 influence-matrix
    columns computed by __cuda on the GPU, against the same rebuild over the
    reference __interaction and against the golden strengths."""
    d = load("vring1_resolve")
    n = d["strengths"].size
    gpu, cpu = np.empty(n), np.empty(n)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        os.chdir(tmp)
        try:
            st = lib.dropin_vring_resolve(float(d["radius"]), float(d["core"]), int(d["layers"]),
                                          gpu.ctypes.data_as(_dp), cpu.ctypes.data_as(_dp))
        finally:
            os.chdir(cwd)
    assert st == 0
    assert np.array_equal(cpu, d["strengths"])
    # an LU solve of a matrix whose entries agree to ~1e-15
    assert rms_rel(gpu, cpu) < 1e-10 and max_rel(gpu, cpu) < 1e-10


def _in_data_dir(fn):
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        os.chdir(tmp)
        try:
            return fn()
        finally:
            os.chdir(cwd)


@needs_lib
@pytest.mark.parametrize("radius,core,layers", [(1.0, 0.1, 1), (1.0, 0.1, 2)])
def test_dropin_batched_resolve_matches_reference_rebuild(lib, radius, core, layers):
    """__cuda_resolve::rebuild (all (2L+1)^2 influence columns in one device
    call) against the reference's __resolve::rebuild over the same __cuda (one
    solve per column): the same resolved strengths bit for bit and a
    byte-identical .wakeinfluence file.  layers = 2 is the vring the
    reference's main() resolves (25 columns, 3,950 particles)."""
    n = (2 * layers + 1) ** 2
    b, p = np.empty(n), np.empty(n)
    same = ctypes.c_int(0)
    st = _in_data_dir(lambda: lib.dropin_vring_resolve_batched(
        radius, core, layers, b.ctypes.data_as(_dp), p.ctypes.data_as(_dp), ctypes.byref(same)))
    assert st == 0
    assert same.value == 1
    assert np.array_equal(b, p)
    if layers == 1:
        d = load("vring1_resolve")
        assert float(d["radius"]) == radius and float(d["core"]) == core and int(d["layers"]) == 1
        assert rms_rel(b, d["strengths"]) < 1e-10 and max_rel(b, d["strengths"]) < 1e-10
