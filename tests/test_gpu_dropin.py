"""The drop-in classes inside the reference's own object model: pawan::__cuda
(a sibling of __parallel) and pawan::__cuda_rk4, built with the reference's
compiled sources into oracle/_ref/libpawan_dropin.so, driven by the reference's
__rk4 / __integration exactly as its main() would."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from pawan_b200 import geometry as g
from helpers import TOL_F32_RMS, load, rms_rel

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libpawan_dropin.so")
needs_lib = pytest.mark.skipif(not os.path.exists(LIB), reason="drop-in harness not built")

_dp = ctypes.POINTER(ctypes.c_double)
_szp = ctypes.POINTER(ctypes.c_size_t)


@pytest.fixture(scope="module")
def lib():
    L = ctypes.CDLL(LIB)
    base = [ctypes.c_int, _szp, _dp, _dp, _dp, _dp]
    L.dropin_solve.argtypes = base + [ctypes.c_double, ctypes.c_int, _dp, _dp]
    L.dropin_rk4.argtypes = base + [ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_size_t,
                                    ctypes.c_int, _dp]
    L.dropin_diagnose.argtypes = base + [_dp, _dp]
    L.dropin_integrate.argtypes = base + [ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_size_t]
    return L


def args(sc):
    pos, vor, rad, vol = (np.ascontiguousarray(a) for a in sc.union())
    cnt = np.asarray(sc.counts, dtype=np.uintp)
    keep = (cnt, pos, vor, rad, vol)
    return keep, [len(sc.counts), cnt.ctypes.data_as(_szp)] + [a.ctypes.data_as(_dp) for a in (pos, vor, rad, vol)]


@needs_lib
@pytest.mark.parametrize("prec,t", [(0, TOL_F32_RMS), (2, 1e-12)])
def test_cuda_solve_matches_reference_interaction(lib, prec, t):
    sc = g.ring_pair(n_stations=24, seed=41, nu=1e-3)
    keep, a = args(sc)
    gpu, cpu = np.empty(6 * sc.n), np.empty(6 * sc.n)
    assert lib.dropin_solve(*a, sc.nu, prec, gpu.ctypes.data_as(_dp), cpu.ctypes.data_as(_dp)) == 0
    assert rms_rel(gpu, cpu) <= t
    assert rms_rel(gpu[:3 * sc.counts[0]], cpu[:3 * sc.counts[0]]) <= t


@needs_lib
def test_reference_rk4_drives_cuda_and_device_rk4_agrees(lib):
    sc = g.ring_pair(n_stations=16, seed=42, nu=1e-3)
    keep, a = args(sc)
    out = {}
    for mode in (0, 1, 2):
        st = sc.state().copy()
        assert lib.dropin_rk4(*a, sc.nu, 2, 0.005, 3, mode, st.ctypes.data_as(_dp)) == 0
        out[mode] = st
    st0 = sc.state()
    # reference __rk4 on __cuda (host path) and __cuda_rk4 (device path) against
    # the reference __rk4 on __interaction, FP64 pair kernel
    assert rms_rel(out[0] - st0, out[2] - st0) < 1e-11
    assert rms_rel(out[1] - st0, out[2] - st0) < 1e-11


@needs_lib
def test_cuda_diagnose_matches_reference(lib):
    d = load("pair64_diag")
    sc_counts = [int(c) for c in d["counts"]]
    cnt = np.asarray(sc_counts, dtype=np.uintp)
    arrs = [np.ascontiguousarray(d[k]) for k in ("pos", "vor", "rad", "vol")]
    gpu, cpu = np.zeros(11), np.zeros(11)
    assert lib.dropin_diagnose(len(sc_counts), cnt.ctypes.data_as(_szp), *[x.ctypes.data_as(_dp) for x in arrs],
                               gpu.ctypes.data_as(_dp), cpu.ctypes.data_as(_dp)) == 0
    assert abs(gpu[9] / cpu[9] - 1) < 1e-12
    assert abs(gpu[10] - cpu[10]) < 1e-10 * abs(cpu[9])
    assert np.abs(gpu[:3] - cpu[:3]).max() < 1e-14 * np.abs(d["vor"]).sum()


@needs_lib
def test_integrate_writes_reference_wake_file(lib):
    d = load("ring16_integrate")
    cnt = np.asarray([int(c) for c in d["counts"]], dtype=np.uintp)
    arrs = [np.ascontiguousarray(d[k]) for k in ("pos", "vor", "rad", "vol")]
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        os.chdir(tmp)
        try:
            rc = lib.dropin_integrate(len(cnt), cnt.ctypes.data_as(_szp), *[x.ctypes.data_as(_dp) for x in arrs],
                                      0.0, 2, float(d["T"]), int(d["nsteps"]))
        finally:
            os.chdir(cwd)
        assert rc == 0
        raw = open(os.path.join(tmp, "data", "temp.wake"), "rb").read()
    ref = d["wake_bytes"].tobytes()
    assert len(raw) == len(ref)
    assert np.allclose(np.frombuffer(raw, np.float64), np.frombuffer(ref, np.float64), rtol=1e-12, atol=1e-15)


@needs_lib
@pytest.mark.parametrize("mode", [0, 1])
def test_integrate_host_and_device_loops_write_the_reference_file(lib, mode):
    """__cuda_rk4 through an __integration reference (the reference's own
    integrate() loop, frames from the wakes) and through __cuda_rk4::integrate
    (device loop, frames written asynchronously): both files match the one the
    reference's integrate() wrote (layout exactly, values to FP64 rounding)."""
    lib.dropin_integrate2.argtypes = [ctypes.c_int, _szp, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_size_t, ctypes.c_int]
    d = load("ring16_integrate")
    cnt = np.asarray([int(c) for c in d["counts"]], dtype=np.uintp)
    arrs = [np.ascontiguousarray(d[k]) for k in ("pos", "vor", "rad", "vol")]
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        os.chdir(tmp)
        try:
            rc = lib.dropin_integrate2(len(cnt), cnt.ctypes.data_as(_szp), *[x.ctypes.data_as(_dp) for x in arrs],
                                       0.0, 2, float(d["T"]), int(d["nsteps"]), mode)
        finally:
            os.chdir(cwd)
        assert rc == 0
        raw = open(os.path.join(tmp, "data", "temp.wake"), "rb").read()
    ref = d["wake_bytes"].tobytes()
    assert len(raw) == len(ref)
    a, b = np.frombuffer(raw, np.uint64), np.frombuffer(ref, np.uint64)
    n = int(d["counts"].sum())
    frame = 3 + 7 * n
    for k in range(int(d["nsteps"]) + 1):  # nWake and N words are integers: exact
        assert a[k * frame + 1] == b[k * frame + 1] and a[k * frame + 2] == b[k * frame + 2]
    assert np.allclose(np.frombuffer(raw, np.float64)[0::frame], np.frombuffer(ref, np.float64)[0::frame])
    assert np.allclose(np.frombuffer(raw, np.float64), np.frombuffer(ref, np.float64), rtol=1e-12, atol=1e-15)
