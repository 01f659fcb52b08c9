"""The allocation-free solve (pawan_interact_noalloc), through the C ABI.

It exists for callers that cannot let a library call cudaMalloc: code running
in a host callback, under an allocator that owns all device memory, or in a
loop where an allocation's implicit device synchronisation is not acceptable.
It keeps its working memory in one static device array and takes caller-owned
device buffers.

Checked here: two calls in a row (different inputs, so nothing left in the
shared array from the first call can leak into the second) each agree with
the allocating entry point (pawan_system_solve, FP32) and with the FP64
oracle within the FP32 tolerance used throughout the tests; a call on a
stream the test creates; a call at exactly the array's particle limit; and
sizes beyond the limit, or a non-finite nu, are rejected without running
anything.  This file is collected last so that a stop-at-first-failure run
has already run every other test.
"""
import numpy as np
import pytest
import torch

import oracle
import pawan_b200
from pawan_b200 import System, interact_noalloc
from pawan_b200 import geometry as g
from helpers import TOL_F32_MAX, TOL_F32_RMS, max_rel, rms_rel

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def run_noalloc(sc, stream=None):
    pos, vor, rad, vol = (dev(a) for a in sc.union())
    vel = torch.empty((sc.n, 3), dtype=torch.float64, device="cuda")
    dvor = torch.empty((sc.n, 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    handle = stream.cuda_stream if stream is not None else 0
    st = interact_noalloc(pos.data_ptr(), vor.data_ptr(), rad.data_ptr(), vol.data_ptr(), sc.n, sc.nu,
                          vel.data_ptr(), dvor.data_ptr(), handle)
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    assert st == 0
    return vel.cpu().numpy(), dvor.cpu().numpy()


def run_allocating(ctx, sc):
    s = System.from_scenario(ctx, sc, "f32")
    s.solve()
    out = s.union_rates()
    s.close()
    return out


def within_f32(u, da, u_ref, da_ref):
    assert np.isfinite(u).all() and np.isfinite(da).all()
    assert rms_rel(u, u_ref) <= TOL_F32_RMS and rms_rel(da, da_ref) <= TOL_F32_RMS, \
        (rms_rel(u, u_ref), rms_rel(da, da_ref))
    assert max_rel(u, u_ref) <= TOL_F32_MAX and max_rel(da, da_ref) <= TOL_F32_MAX, \
        (max_rel(u, u_ref), max_rel(da, da_ref))


def test_noalloc_matches_allocating_entry_point_twice(ctx):
    first = g.ring_pair(n_stations=640, seed=71, nu=1e-4)        # N = 10,240, diffusion on
    second = g.helical_wake(n_stations=64, seed=72, turns=2.0)   # N = 2,048, four wakes
    second.nu = 0.0
    for sc in (first, second):
        u, da = run_noalloc(sc)
        within_f32(u, da, *run_allocating(ctx, sc))
        # and against the FP64 oracle (sampled targets, summed over all sources)
        t = np.sort(np.random.default_rng(sc.n).choice(sc.n, 512, replace=False))
        pos, vor, rad, vol = sc.union()
        u_or, da_or = oracle.pairs(pos, vor, rad, vol, sc.nu, targets=t)
        within_f32(u[t], da[t], u_or, da_or)
    # repeated call on the same inputs: identical bits
    a = run_noalloc(second)
    b = run_noalloc(second)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_noalloc_on_a_created_stream_at_the_particle_limit(ctx):
    """N = PAWAN_NOALLOC_MAX_PARTICLES exactly (every partial and item slot of
    the array in use), called on a non-default stream, twice."""
    n_st = pawan_b200.NOALLOC_MAX_PARTICLES // 16   # two rings x n_st stations x 8
    sc = g.ring_pair(n_stations=n_st, seed=73, nu=2e-4)
    assert sc.n == pawan_b200.NOALLOC_MAX_PARTICLES
    stream = torch.cuda.Stream()
    u, da = run_noalloc(sc, stream)
    within_f32(u, da, *run_allocating(ctx, sc))
    u2, da2 = run_noalloc(sc, stream)
    assert np.array_equal(u, u2) and np.array_equal(da, da2)
    # the default stream gives the same bits
    u3, da3 = run_noalloc(sc)
    assert np.array_equal(u, u3) and np.array_equal(da, da3)


def test_noalloc_rejects_sizes_beyond_its_array():
    n = pawan_b200.NOALLOC_MAX_PARTICLES + 1
    buf = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert interact_noalloc(p, p, p, p, n, 0.0, p, p, 0) == 1  # PAWAN_ERR_INVALID
    assert interact_noalloc(p, p, p, p, 1, 0.0, p, p, 0) == 1
    assert interact_noalloc(p, p, p, p, 8, float("inf"), p, p, 0) == 1
    assert interact_noalloc(p, p, p, p, 8, float("nan"), p, p, 0) == 1
    assert interact_noalloc(p, p, p, p, 8, -1e-3, p, p, 0) == 1
    torch.cuda.synchronize()
