"""The oracle's host code under AddressSanitizer and UndefinedBehaviorSanitizer
(compute-sanitizer is not available for the GPU side): the reference's own
sources on the GSL shim, the harness and the C restatement, built by
`make -C oracle sanitize` and driven by oracle/sanitize_main.cpp on a small
ring pair, the OpenMP path, RK4, Euler, diagnostics, the vorticity field and
the vring resolve.  CPU only; needs the reference tree to build."""
import os
import subprocess
import tempfile

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_tree() -> str:
    """The reference tree: $PAWAN_REF (as `make REF=...` takes it), else the
    oracle Makefile's own default."""
    if os.environ.get("PAWAN_REF"):
        return os.environ["PAWAN_REF"]
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s", "--no-print-directory",
                        "print-ref"], capture_output=True, text=True)
    return r.stdout.strip() if r.returncode == 0 else ""


REF = _reference_tree()
needs_tree = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")),
                                reason="reference tree absent")


@needs_tree
def test_oracle_host_code_is_clean_under_asan_and_ubsan():
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s", f"REF={REF}", "sanitize"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    exe = os.path.join(ROOT, "oracle", "_ref", "sanitize_check")
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1",
               UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1", OMP_NUM_THREADS="2")
    with tempfile.TemporaryDirectory() as tmp:
        # the reference's __io writes data/temp.* and does not create data/
        os.makedirs(os.path.join(tmp, "data"))
        r = subprocess.run([exe], cwd=tmp, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "sanitized oracle run ok" in r.stdout
