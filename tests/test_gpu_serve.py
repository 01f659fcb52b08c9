"""The continuous-batching serving loop: results alone vs in the mix,
admission by memory budget, queue limits, cancellation."""
import time

import numpy as np
import pytest

from pawan_b200 import Server, System
from pawan_b200 import geometry as g
from helpers import TOL_F32_RMS, rms_rel

pytestmark = pytest.mark.gpu


def requests(k=5, seed=7):
    reqs = g.serving_requests(rate=1000.0, duration=1.0, seed=seed, n_lo=64, n_hi=1200,
                              steps_lo=2, steps_hi=6)
    return [r.scenario for r in reqs[:k]]


def run_alone(ctx, sc):
    srv = Server(ctx, budget_bytes=1 << 30)
    st, rid = srv.submit_scenario(sc)
    assert st == 0
    assert srv.wait(rid, 60)
    out, *_ = srv.fetch(rid)
    srv.close()
    return out


def test_alone_and_in_the_mix_are_identical(ctx):
    scs = requests()
    # a tiny iteration target: requests advance a slice of a step per iteration,
    # so the staggered arrivals join requests in flight
    srv = Server(ctx, budget_bytes=1 << 30, iteration_seconds=1e-9)
    ids = []
    for k, sc in enumerate(scs):
        st, rid = srv.submit_scenario(sc)
        assert st == 0
        ids.append(rid)
        time.sleep(0.002 * k)  # staggered arrivals join running iterations
    for rid in ids:
        assert srv.wait(rid, 120)
    mixed = [srv.fetch(rid) for rid in ids]
    stats = srv.stats()
    tiling = srv.tiling()
    srv.close()
    assert stats["completed"] == len(scs) and stats["rejected"] == 0
    for sc, (out, ts, ta, td) in zip(scs, mixed):
        assert out is not None and ts <= ta <= td
        alone = run_alone(ctx, sc)
        assert np.array_equal(out, alone)
        # a system of its own with the engine's tiling: the same FP32 tile sums,
        # grouped differently in FP64
        solo = System.from_scenario(ctx, sc, "f32")
        solo.set_config(**tiling)
        solo.rk4(sc.dt, sc.steps)
        st0 = sc.state()
        assert rms_rel(out - st0, solo.get_states() - st0) < 1e-12
    # at least one request was admitted while another was still running
    spans = [(ta, td) for _, ts, ta, td in mixed]
    assert any(a2 < d1 and a1 <= a2 for i, (a1, d1) in enumerate(spans)
               for j, (a2, d2) in enumerate(spans) if i != j)


def test_multi_step_iterations_match_single_steps(ctx):
    """The default policy runs several RK4 steps per iteration (CUDA-graph
    replays); every request's result is bit-identical to one step per
    iteration, and all requests finish."""
    reqs = g.serving_requests(rate=1000.0, duration=1.0, seed=9, n_lo=64, n_hi=1500,
                              steps_lo=10, steps_hi=40)
    scs = [r.scenario for r in reqs[:8]]
    outs = []
    for target in (0.0, 1e-9):
        srv = Server(ctx, budget_bytes=1 << 30, iteration_seconds=target)
        ids = [srv.submit_scenario(sc)[1] for sc in scs]
        for rid in ids:
            assert srv.wait(rid, 120)
        outs.append([srv.fetch(rid)[0] for rid in ids])
        stats = srv.stats()
        srv.close()
        assert stats["completed"] == len(scs)
        if target == 0.0:
            # fewer iterations than the longest request has steps
            assert stats["iterations"] < max(sc.steps for sc in scs)
    for a, b in zip(*outs):
        assert a is not None and np.array_equal(a, b)


def test_budget_rejects_oversized_request(ctx):
    srv = Server(ctx, budget_bytes=1e5)
    sc = g.single_ring(n_stations=64, seed=1)
    st, rid = srv.submit_scenario(sc, nsteps=1)
    assert st == 5  # exceeds budget
    assert srv.poll(rid) == "rejected"
    srv.close()


def test_budget_serialises_admission(ctx):
    """A budget that fits one request at a time: all finish, never two active."""
    scs = [g.single_ring(n_stations=128, seed=s, steps=3) for s in (1, 2, 3)]
    probe = Server(ctx, budget_bytes=1 << 30)
    rid = probe.submit_scenario(scs[0], nsteps=10_000_000)[1]  # cancelled below
    while probe.poll(rid) == "queued":
        time.sleep(0.001)
    one = probe.stats()["bytes_in_use"]
    probe.cancel(rid)
    probe.close()
    assert one > 0
    srv = Server(ctx, budget_bytes=one * 1.5)
    ids = [srv.submit_scenario(sc)[1] for sc in scs]
    peak_active = 0
    deadline = time.time() + 120
    while time.time() < deadline:
        s = srv.stats()
        peak_active = max(peak_active, s["active"])
        if s["completed"] == len(scs):
            break
        time.sleep(0.001)
    assert srv.stats()["completed"] == len(scs)
    assert peak_active <= 1
    for rid in ids:
        out, *_ = srv.fetch(rid)
        assert out is not None
    srv.close()


def test_queue_limit_and_cancel(ctx):
    sc = g.single_ring(n_stations=64, seed=2)
    srv = Server(ctx, budget_bytes=1 << 30, max_active=1, max_queue=2)
    ids, sts = [], []
    for _ in range(6):
        st, rid = srv.submit_scenario(sc, nsteps=200)
        ids.append(rid)
        sts.append(st)
    assert sts.count(8) >= 1  # queue full -> rejected
    queued = [rid for rid, st in zip(ids, sts) if st == 0 and srv.poll(rid) == "queued"]
    if queued:
        srv.cancel(queued[-1])
        assert srv.poll(queued[-1]) == "cancelled"
    for rid, st in zip(ids, sts):
        if st == 0:
            srv.cancel(rid)
    for rid, st in zip(ids, sts):
        if st == 0:
            assert srv.wait(rid, 60)
    srv.close()


def test_injected_allocation_failure_rejects_one_request(ctx):
    """A failed device allocation at admission (made on the host) rejects that
    request only; the others complete with the same results as alone."""
    scs = requests(k=3, seed=11)
    srv = Server(ctx, budget_bytes=1 << 30)
    srv.inject("alloc", 1)
    ids = [srv.submit_scenario(sc)[1] for sc in scs]
    for rid in ids:
        assert srv.wait(rid, 60)
    states = [srv.poll(rid) for rid in ids]
    assert states.count("rejected") == 1 and states.count("done") == 2
    outs = [srv.fetch(rid)[0] for rid in ids]
    srv.close()
    for sc, out, st in zip(scs, outs, states):
        if st == "done":
            assert np.array_equal(out, run_alone(ctx, sc))
        else:
            assert out is None


def test_injected_iteration_failure_then_recovery(ctx):
    """A failed iteration rejects the requests active in it; the engine then
    serves new requests normally."""
    sc = g.single_ring(n_stations=64, seed=12, steps=5)
    srv = Server(ctx, budget_bytes=1 << 30, iteration_seconds=1e-9)
    srv.inject("iteration", 1)
    rid = srv.submit_scenario(sc)[1]
    assert srv.wait(rid, 60)
    assert srv.poll(rid) == "rejected"
    rid2 = srv.submit_scenario(sc)[1]
    assert srv.wait(rid2, 60)
    assert srv.poll(rid2) == "done"
    out, *_ = srv.fetch(rid2)
    srv.close()
    assert np.array_equal(out, run_alone(ctx, sc))


def test_injected_slow_iteration_times_out_the_wait(ctx):
    """A slow iteration: a short wait times out, a longer one completes."""
    sc = g.single_ring(n_stations=32, seed=13, steps=2)
    srv = Server(ctx, budget_bytes=1 << 30)
    srv.inject("slow", 1, seconds=1.0)
    rid = srv.submit_scenario(sc)[1]
    assert srv.wait(rid, 0.2) is False
    assert srv.wait(rid, 30)
    assert srv.poll(rid) == "done"
    srv.close()


@pytest.mark.parametrize("policy", ["fifo", "shortest"])
def test_admission_policy_orders_the_queue(ctx, policy):
    """One request at a time: while the first runs, a large and then a small
    request wait; FIFO admits the large one next, shortest-first the small one.
    Results are the same under either policy."""
    srv = Server(ctx, budget_bytes=1 << 30, max_active=1, iteration_seconds=1e-9, policy=policy)
    first = g.single_ring(n_stations=64, seed=21, steps=300)
    big = g.single_ring(n_stations=256, seed=22, steps=20)
    small = g.single_ring(n_stations=32, seed=23, steps=5)
    ra = srv.submit_scenario(first)[1]
    deadline = time.time() + 30
    while srv.poll(ra) == "queued" and time.time() < deadline:
        time.sleep(0.0005)
    rb = srv.submit_scenario(big)[1]
    rc = srv.submit_scenario(small)[1]
    for rid in (ra, rb, rc):
        assert srv.wait(rid, 120)
    outs = {rid: srv.fetch(rid) for rid in (ra, rb, rc)}
    srv.close()
    t_admit_big, t_admit_small = outs[rb][2], outs[rc][2]
    if policy == "fifo":
        assert t_admit_big < t_admit_small
    else:
        assert t_admit_small < t_admit_big
    assert np.array_equal(outs[rc][0], run_alone(ctx, small))


def test_large_requests_advance_by_slices_with_identical_results(ctx):
    """With a tiny iteration target every request is "large": each advances by
    slices of its stages' work items over many iterations.  Results are
    bit-identical to one request alone with the ordinary path."""
    scs = requests(k=3, seed=31)
    srv = Server(ctx, budget_bytes=1 << 30, iteration_seconds=1e-7)
    ids = [srv.submit_scenario(sc)[1] for sc in scs]
    for rid in ids:
        assert srv.wait(rid, 120)
    outs = [srv.fetch(rid)[0] for rid in ids]
    stats = srv.stats()
    srv.close()
    assert stats["completed"] == len(scs)
    assert stats["iterations"] > 4 * sum(sc.steps for sc in scs) / len(scs)  # stages split up
    for sc, out in zip(scs, outs):
        assert np.array_equal(out, run_alone(ctx, sc))


def test_small_requests_keep_their_pace_beside_a_large_one(ctx):
    """A large request (one step far beyond the iteration target) does not hold
    the small ones: they finish while it is still running."""
    srv = Server(ctx, budget_bytes=8 << 30, iteration_seconds=0.002)
    big = g.ring_pair(n_stations=2048, seed=32, steps=50)        # N = 32,768
    rb = srv.submit_scenario(big)[1]
    deadline = time.time() + 30
    while srv.poll(rb) == "queued" and time.time() < deadline:
        time.sleep(0.001)
    small = [g.single_ring(n_stations=32, seed=33 + i, steps=5) for i in range(4)]
    ids = [srv.submit_scenario(sc)[1] for sc in small]
    for rid in ids:
        assert srv.wait(rid, 60)
    assert srv.poll(rb) == "active"
    outs = [srv.fetch(rid)[0] for rid in ids]
    srv.cancel(rb)
    srv.close()
    for sc, out in zip(small, outs):
        assert np.array_equal(out, run_alone(ctx, sc))
