"""Shared test helpers: error metrics with the stated tolerances, golden fixtures."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Stated tolerances (relative to the FP64 reference values):
#   FP32 pair math with FP64 accumulation: RMS relative error <= 1e-5,
#     max-abs error / max-abs reference <= 1e-4;
#   plain FP64 (the reference's formula term by term): RMS <= 1e-12, max <= 1e-11;
#   tuned FP64 (rsqrt algebra, FMA): RMS <= 1e-10, max <= 1e-9.  The stretching
#     term F [d.(alpha_i x alpha_j)] d is a triple product that nearly vanishes
#     for a flat ring, so the reference's own FP64 value is only accurate to
#     ~1e-16 / flatness there; a different (equally valid) rounding order
#     disagrees with it at that level.
TOL_F32_RMS = 1e-5
TOL_F32_MAX = 1e-4
TOL_F64_RMS = 1e-12
TOL_F64_MAX = 1e-11
TOL_F64T_RMS = 1e-10
TOL_F64T_MAX = 1e-9


from pawan_b200 import max_rel, rms_rel  # noqa: F401  (the metrics the bench reports too)


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def split_rates(counts, rates):
    """Reference rate vector -> (u, dalpha) union arrays."""
    us, das, o = [], [], 0
    for c in counts:
        blk = rates[6 * o: 6 * (o + c)]
        us.append(blk[:3 * c].reshape(c, 3))
        das.append(blk[3 * c:].reshape(c, 3))
        o += c
    return np.concatenate(us), np.concatenate(das)


def tol(precision):
    return {"f32": (TOL_F32_RMS, TOL_F32_MAX), "f64": (TOL_F64T_RMS, TOL_F64T_MAX),
            "f64_plain": (TOL_F64_RMS, TOL_F64_MAX)}[precision]
