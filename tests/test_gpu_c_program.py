"""The C ABI from a plain C program (tests/abi/solve_file.c, compiled here
with gcc against include/pawan_b200.h and the built library; no Python in
the loop): solve and RK4 of a two-wake system against the reference's own
outputs (golden fixtures), FP32 and plain FP64."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from pawan_b200 import LIB_PATH
from helpers import TOL_F32_RMS, TOL_F64_RMS, load, rms_rel

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("abi") / "solve_file")
    libdir = os.path.dirname(LIB_PATH)
    r = subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "abi", "solve_file.c"), "-L", libdir, "-lpawan_b200",
                        f"-Wl,-rpath,{libdir}", "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def run(program, d, precision, nsteps, dt):
    n = int(d["counts"].sum())
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            np.array([len(d["counts"])], dtype=np.int64).tofile(f)
            d["counts"].astype(np.int64).tofile(f)
            np.array([float(d["nu"])]).tofile(f)
            for k in ("pos", "vor", "rad", "vol"):
                np.ascontiguousarray(d[k], dtype=np.float64).tofile(f)
        r = subprocess.run([program, fin, fout, str(precision), str(nsteps), repr(dt)],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        out = np.fromfile(fout, dtype=np.float64)
    return out[:6 * n], out[6 * n:]


@pytest.mark.parametrize("precision,tol", [(0, TOL_F32_RMS), (2, TOL_F64_RMS)])
def test_c_program_solve_and_rk4(program, precision, tol):
    d = load("pair64_solve")
    rates, _ = run(program, d, precision, 0, 0.0)
    assert rms_rel(rates, d["rates"]) < tol
    r = load("pair64_rk4")
    _, state = run(program, r, precision, int(r["nsteps"]), float(r["dt"]))
    assert rms_rel(state - r["state"], r["final_state"] - r["state"]) < (1e-5 if precision == 0 else 1e-11)
