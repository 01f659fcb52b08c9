"""Test infrastructure: the parity oracle.

Two CPU libraries, both used only as checkers (by tests/, the smoke check and
bench.py's CPU-baseline leg), never as the product:

* ``_ref/libpawan_ref.so`` -- the reference's own C++ classes (``__wake``,
  ``__interaction``, ``__parallel``, ``__rk4``), compiled from their unmodified
  sources against the project's GSL-API shim by ``oracle/Makefile``.
* ``liboracle.so`` -- the project's plain-C FP64 restatement (``restate.c``),
  checked against the compiled reference in ``tests/test_oracle.py`` and used
  where running the reference would take too long.

Arrays are float64, C-contiguous; a "system" is the union of its wakes in
wake order with positions/vorticities N x 3.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libpawan_ref.so")
# the same reference sources compiled with their Gaussian smoothing kernel
REF_GAUSS_LIB = os.path.join(_HERE, "_ref", "libpawan_ref_gauss.so")
KERNELS = {"highorder": 0, "gaussian": 1}
RESTATE_LIB = os.path.join(_HERE, "liboracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_szp = ctypes.POINTER(ctypes.c_size_t)


def _ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


_ref = {}
_orc = None


def ref_available(kernel: str = "highorder") -> bool:
    return os.path.exists(REF_GAUSS_LIB if kernel == "gaussian" else REF_LIB)


def _load_ref(kernel: str = "highorder"):
    if kernel not in _ref:
        path = REF_GAUSS_LIB if kernel == "gaussian" else REF_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle)")
        lib = ctypes.CDLL(path)
        lib.refh_create.restype = ctypes.c_void_p
        lib.refh_create.argtypes = [ctypes.c_int, _szp, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int]
        lib.refh_destroy.argtypes = [ctypes.c_void_p]
        lib.refh_size.restype = ctypes.c_size_t
        lib.refh_size.argtypes = [ctypes.c_void_p]
        for name in ("refh_set_states", "refh_get_states", "refh_get_rates"):
            getattr(lib, name).argtypes = [ctypes.c_void_p, _dp]
        lib.refh_solve.argtypes = [ctypes.c_void_p]
        lib.refh_get_wake_rates.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        lib.refh_rk4_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_size_t, _dp]
        lib.refh_euler_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_size_t, _dp]
        lib.refh_integrate.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_size_t]
        lib.refh_diagnose.restype = ctypes.c_int
        lib.refh_diagnose.argtypes = [ctypes.c_void_p, _dp]
        lib.refh_kinetic_energy.restype = ctypes.c_double
        lib.refh_kinetic_energy.argtypes = [ctypes.c_void_p]
        lib.refh_write_frame.restype = ctypes.c_int
        lib.refh_write_frame.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_int]
        lib.refh_vring_create.restype = ctypes.c_void_p
        lib.refh_vring_create.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double]
        lib.refh_num_particles.restype = ctypes.c_size_t
        lib.refh_num_particles.argtypes = [ctypes.c_void_p]
        lib.refh_get_particles.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
        lib.refh_influence.argtypes = [ctypes.c_void_p, _dp]
        lib.refh_resolve.argtypes = [ctypes.c_void_p, _dp]
        lib.refh_set_threads.argtypes = [ctypes.c_int]
        lib.refh_max_threads.restype = ctypes.c_int
        lib.refh_wtime.restype = ctypes.c_double
        _ref[kernel] = lib
    return _ref[kernel]


def _load_orc():
    global _orc
    if _orc is None:
        if not os.path.exists(RESTATE_LIB):
            raise FileNotFoundError(f"{RESTATE_LIB} not built (make -C oracle)")
        lib = ctypes.CDLL(RESTATE_LIB)
        lib.orc_pairs.argtypes = [ctypes.c_size_t, _dp, _dp, _dp, _dp, ctypes.c_double,
                                  ctypes.c_size_t, _i64p, _dp, _dp]
        lib.orc_rk4_step.argtypes = [ctypes.c_size_t, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double]
        lib.orc_linear_diagnostics.argtypes = [ctypes.c_size_t, _dp, _dp, _dp]
        for name in ("orc_enstrophy", "orc_helicity"):
            getattr(lib, name).restype = ctypes.c_double
            getattr(lib, name).argtypes = [ctypes.c_size_t, _dp, _dp, _dp]
        lib.orc_influence.argtypes = [ctypes.c_size_t, _dp, _dp, _dp, _dp]
        lib.orc_set_kernel.argtypes = [ctypes.c_int]
        lib.orc_kinetic_energy.restype = ctypes.c_double
        lib.orc_kinetic_energy.argtypes = [ctypes.c_size_t, _i32p, _dp, _dp, _dp]
        _orc = lib
    return _orc


class RefSystem:
    """The reference's ``__interaction`` (serial) or ``__parallel`` (OpenMP)
    over wakes built from arrays, with viscosity ``nu``."""

    def __init__(self, counts: Sequence[int], pos, vor, rad, vol, nu: float, parallel: bool = False,
                 kernel: str = "highorder"):
        lib = _load_ref(kernel)
        self._lib = lib
        self.counts = [int(c) for c in counts]
        self.n = sum(self.counts)
        pos, vor, rad, vol = _f64(pos), _f64(vor), _f64(rad), _f64(vol)
        cnt = np.asarray(self.counts, dtype=np.uintp)
        self._h = lib.refh_create(len(self.counts), cnt.ctypes.data_as(_szp), _ptr(pos), _ptr(vor),
                                  _ptr(rad), _ptr(vol), float(nu), 1 if parallel else 0)
        self.parallel = parallel
        self.size = lib.refh_size(self._h)

    def close(self):
        if self._h:
            self._lib.refh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_states(self, state):
        s = _f64(state)
        assert s.size == self.size
        self._lib.refh_set_states(self._h, _ptr(s))

    def get_states(self) -> np.ndarray:
        s = np.empty(self.size)
        self._lib.refh_get_states(self._h, _ptr(s))
        return s

    def solve(self):
        self._lib.refh_solve(self._h)

    def get_rates(self) -> np.ndarray:
        r = np.empty(self.size)
        self._lib.refh_get_rates(self._h, _ptr(r))
        return r

    def wake_rates(self, w: int):
        n = self.counts[w]
        u, da = np.empty((n, 3)), np.empty((n, 3))
        self._lib.refh_get_wake_rates(self._h, w, _ptr(u), _ptr(da))
        return u, da

    def union_rates(self):
        us, das = zip(*(self.wake_rates(w) for w in range(len(self.counts))))
        return np.concatenate(us), np.concatenate(das)

    def rk4(self, state, dt: float, nsteps: int = 1) -> np.ndarray:
        s = _f64(state).copy()
        self._lib.refh_rk4_step(self._h, float(dt), int(nsteps), _ptr(s))
        return s

    def euler(self, state, dt: float, nsteps: int = 1) -> np.ndarray:
        s = _f64(state).copy()
        self._lib.refh_euler_step(self._h, float(dt), int(nsteps), _ptr(s))
        return s

    def integrate(self, T: float, n: int):
        self._lib.refh_integrate(self._h, float(T), int(n))

    def diagnose(self) -> dict:
        out = np.zeros(11)
        if self._lib.refh_diagnose(self._h, _ptr(out)) != 0:
            raise RuntimeError("diagnostics are taken from the serial system only")
        return {"total_vorticity": out[0:3].copy(), "linear_impulse": out[3:6].copy(),
                "angular_impulse": out[6:9].copy(), "enstrophy": float(out[9]),
                "helicity": float(out[10])}

    def kinetic_energy(self) -> float:
        return float(self._lib.refh_kinetic_energy(self._h))

    def write_frame(self, path: str, t: float, append: bool):
        if self._lib.refh_write_frame(self._h, path.encode(), float(t), 1 if append else 0) != 0:
            raise OSError(f"cannot open {path}")

    def influence(self) -> np.ndarray:
        """__interaction::resolve() -> influence(): the vorticity field (N x 3)."""
        k = np.empty((self._lib.refh_num_particles(self._h), 3))
        self._lib.refh_influence(self._h, _ptr(k))
        return k

    def particles(self):
        """(pos, vor, rad, vol) of the wakes, union order."""
        n = self._lib.refh_num_particles(self._h)
        pos, vor, rad, vol = np.empty((n, 3)), np.empty((n, 3)), np.empty(n), np.empty(n)
        self._lib.refh_get_particles(self._h, _ptr(pos), _ptr(vor), _ptr(rad), _ptr(vol))
        return pos, vor, rad, vol

    def resolve(self) -> np.ndarray:
        """__resolve::rebuild on this system (writes data/temp.wakeinfluence in
        the current directory); returns the resolved state."""
        s = np.empty(self.size)
        self._lib.refh_resolve(self._h, _ptr(s))
        return s


class RefVring(RefSystem):
    """The reference's ``__vring(radius, core, layers)`` (src/wake/vring.cpp:51-104)
    in a serial ``__interaction``; its state is the per-layer strength vector."""

    def __init__(self, radius: float, core: float, layers: int, nu: float = 0.0):
        lib = _load_ref()
        self._lib = lib
        self._h = lib.refh_vring_create(float(radius), float(core), int(layers), float(nu))
        self.n = lib.refh_num_particles(self._h)
        self.counts = [self.n]
        self.parallel = False
        self.size = lib.refh_size(self._h)


def ref_set_threads(n: int):
    _load_ref().refh_set_threads(int(n))


def ref_max_threads() -> int:
    return int(_load_ref().refh_max_threads())


def ref_wtime() -> float:
    return float(_load_ref().refh_wtime())


# ----------------------------------------------------------------- restatement

def _restate(kernel: str = "highorder"):
    lib = _load_orc()
    lib.orc_set_kernel(KERNELS[kernel])
    return lib


def pairs(pos, vor, rad, vol, nu: float, targets=None, kernel: str = "highorder"):
    """(velocity, vorticity rate) of `targets` (all when None), FP64."""
    lib = _restate(kernel)
    pos, vor, rad, vol = _f64(pos), _f64(vor), _f64(rad), _f64(vol)
    n = rad.shape[0]
    if targets is None:
        nt, tp = n, None
    else:
        t = np.ascontiguousarray(targets, dtype=np.int64)
        nt, tp = t.shape[0], _ptr(t, _i64p)
    u, da = np.empty((nt, 3)), np.empty((nt, 3))
    lib.orc_pairs(n, _ptr(pos), _ptr(vor), _ptr(rad), _ptr(vol), float(nu), nt, tp, _ptr(u), _ptr(da))
    return u, da


def rk4_step(pos, vor, rad, vol, nu: float, dt: float, nsteps: int = 1, kernel: str = "highorder"):
    lib = _restate(kernel)
    p, v = _f64(pos).copy(), _f64(vor).copy()
    rad, vol = _f64(rad), _f64(vol)
    for _ in range(nsteps):
        lib.orc_rk4_step(rad.shape[0], _ptr(p), _ptr(v), _ptr(rad), _ptr(vol), float(nu), float(dt))
    return p, v


def linear_diagnostics(pos, vor):
    lib = _load_orc()
    pos, vor = _f64(pos), _f64(vor)
    out = np.zeros(9)
    lib.orc_linear_diagnostics(pos.shape[0], _ptr(pos), _ptr(vor), _ptr(out))
    return out[0:3], out[3:6], out[6:9]


def enstrophy(pos, vor, rad, kernel: str = "highorder") -> float:
    pos, vor, rad = _f64(pos), _f64(vor), _f64(rad)
    return float(_restate(kernel).orc_enstrophy(rad.shape[0], _ptr(pos), _ptr(vor), _ptr(rad)))


def helicity(pos, vor, rad, kernel: str = "highorder") -> float:
    pos, vor, rad = _f64(pos), _f64(vor), _f64(rad)
    return float(_restate(kernel).orc_helicity(rad.shape[0], _ptr(pos), _ptr(vor), _ptr(rad)))


def influence(pos, vor, rad, kernel: str = "highorder") -> np.ndarray:
    """Vorticity field K_i = Z(0, s_i) alpha_i + sum_j Z_ij alpha_j (N x 3), FP64."""
    pos, vor, rad = _f64(pos), _f64(vor), _f64(rad)
    k = np.empty((rad.shape[0], 3))
    _restate(kernel).orc_influence(rad.shape[0], _ptr(pos), _ptr(vor), _ptr(rad), _ptr(k))
    return k


def kinetic_energy(wake_id, pos, vor, rad) -> float:
    wid = np.ascontiguousarray(wake_id, dtype=np.int32)
    pos, vor, rad = _f64(pos), _f64(vor), _f64(rad)
    return float(_load_orc().orc_kinetic_energy(rad.shape[0], _ptr(wid, _i32p), _ptr(pos), _ptr(vor), _ptr(rad)))
