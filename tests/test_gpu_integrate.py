"""pawan_system_integrate: the reference's integrate() loop on the device with
the .wake frames written asynchronously.  Checked against the frames of the
reference's own integrate() (golden file), against frames taken one by one
through the synchronous writer after each device step (bit for bit), and read
back in the layout of the reference's reader (scripts/readWake.py:74-114)."""
import os
import tempfile

import numpy as np
import pytest

from pawan_b200 import System, state_to_union
from pawan_b200 import geometry as g
from helpers import load

pytestmark = pytest.mark.gpu


def read_frames(raw, counts):
    """(t, [(N, x, alpha, s) per wake]) per frame."""
    out, off = [], 0
    buf = memoryview(raw)
    while off < len(raw):
        t = np.frombuffer(buf[off:off + 8], np.float64)[0]
        nw = int(np.frombuffer(buf[off + 8:off + 16], np.uint64)[0])
        off += 16
        wakes = []
        for _ in range(nw):
            n = int(np.frombuffer(buf[off:off + 8], np.uint64)[0])
            off += 8
            x = np.frombuffer(buf[off:off + 24 * n], np.float64).reshape(n, 3)
            a = np.frombuffer(buf[off + 24 * n:off + 48 * n], np.float64).reshape(n, 3)
            s = np.frombuffer(buf[off + 48 * n:off + 56 * n], np.float64)
            off += 56 * n
            wakes.append((n, x, a, s))
        out.append((t, wakes))
    return out


def test_integrate_matches_the_reference_file(ctx):
    d = load("ring16_integrate")
    counts = [int(c) for c in d["counts"]]
    s = System(ctx, counts, 0.0, "f64_plain")
    s.set_particles(d["pos"], d["vor"], d["rad"], d["vol"])
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "temp.wake")
        s.integrate(float(d["T"]), int(d["nsteps"]), path)
        raw = open(path, "rb").read()
    ref = d["wake_bytes"].tobytes()
    assert len(raw) == len(ref)
    assert np.allclose(np.frombuffer(raw, np.float64), np.frombuffer(ref, np.float64), rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("method", ["rk4", "euler"])
def test_async_frames_equal_synchronous_frames(ctx, method):
    sc = g.ring_pair(n_stations=64, seed=91, nu=1e-3)  # two wakes, N = 1,024
    T, n = 0.05, 10
    with tempfile.TemporaryDirectory() as tmp:
        a = System.from_scenario(ctx, sc, "f32")
        pa = os.path.join(tmp, "async.wake")
        a.integrate(T, n, pa, method)
        b = System.from_scenario(ctx, sc, "f32")
        pb = os.path.join(tmp, "sync.wake")
        b.write_frame(pb, 0.0, append=False)
        for i in range(1, n + 1):
            (b.rk4 if method == "rk4" else b.euler)(T / n, 1)
            b.write_frame(pb, i * (T / n), append=True)
        ra, rb = open(pa, "rb").read(), open(pb, "rb").read()
        assert ra == rb
        frames = read_frames(ra, sc.counts)
    assert len(frames) == n + 1
    assert [f[0] for f in frames] == [i * (T / n) for i in range(n + 1)]
    t_last, wakes = frames[-1]
    assert [w[0] for w in wakes] == sc.counts
    p, v = state_to_union(sc.counts, a.get_states())
    assert np.array_equal(np.concatenate([w[1] for w in wakes]), p)
    assert np.array_equal(np.concatenate([w[2] for w in wakes]), v)


def test_integrate_reports_an_unwritable_path(ctx):
    sc = g.single_ring(n_stations=8, seed=92)
    s = System.from_scenario(ctx, sc, "f32")
    with pytest.raises(Exception):
        s.integrate(0.01, 1, "/nonexistent-directory/x.wake")
