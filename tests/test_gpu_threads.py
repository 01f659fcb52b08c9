"""Contexts on separate host threads.

The C ABI is used as one context per host thread, each with its own stream;
the library keeps no shared mutable host state besides the per-device kernel
set-up, which is locked.  Four threads each step their own system with their
own context at the same time (ctypes releases the GIL during the calls), and
every result equals the same steps run on one thread, bit for bit (same
tiling, same chunking, hence the same arithmetic).
"""
import threading

import numpy as np
import pytest

from pawan_b200 import Context, System
from pawan_b200 import geometry as g

pytestmark = pytest.mark.gpu


def test_contexts_on_threads_match_one_thread(ctx):
    scs = [g.ring_pair(n_stations=256, seed=40 + k, nu=1e-3) for k in range(4)]  # N = 4,096 each
    ref = []
    for sc in scs:
        s = System.from_scenario(ctx, sc, "f32")
        s.rk4(sc.dt, 3)
        ref.append(s.get_states())
        s.close()

    results = [None] * len(scs)
    errors = []
    start = threading.Barrier(len(scs))

    def work(k):
        try:
            c = Context(0)
            try:
                s = System.from_scenario(c, scs[k], "f32")
                start.wait(timeout=60)
                s.rk4(scs[k].dt, 3)
                results[k] = s.get_states()
                s.close()
            finally:
                c.close()
        except Exception as e:  # reported below, on the test's thread
            errors.append((k, e))

    threads = [threading.Thread(target=work, args=(k,)) for k in range(len(scs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
    for k in range(len(scs)):
        assert np.array_equal(results[k], ref[k]), k
