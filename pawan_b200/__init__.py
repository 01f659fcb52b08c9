"""pawan_b200: B200 (sm_100a) implementation of pawan's hot path.

The compute path is the CUDA library ``pawan_b200/_lib/libpawan_b200.so``
(built by ``python -m pawan_b200.build``), reached through its C ABI
(``include/pawan_b200.h``).  This module is a thin ctypes mirror of the
reference's interface for Python callers and tests:

* :class:`System` -- ``pawan::__interaction`` over its wakes
  (src/interaction/interaction.h:21-235): ``set_states``, ``get_states``,
  ``solve``, ``get_rates``, ``diagnose``, plus the integrators
  ``rk4`` (``__rk4::step``, src/integration/rk4.cpp:12-76) and ``euler``
  (``__integration::step``, src/integration/integration.cpp:37-45).
* :class:`Batch` -- many systems in one persistent launch per RK4 stage.
* :class:`Server` -- the continuous-batching request loop.

There is no CPU fallback: importing works without a GPU (so the library can
be inspected), but creating a :class:`Context` without a B200 raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from . import geometry  # noqa: F401  (seeded workload generators)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libpawan_b200.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "pawan_b200.h")

PREC = {"f32": 0, "f64": 1, "f64_plain": 2}
KERNELS = {"highorder": 0, "gaussian": 1}  # PAWAN_KERNEL_*
OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "cuda error", 3: "out of memory", 4: "invalid state",
          5: "exceeds budget", 6: "timeout", 7: "not found", 8: "rejected"}
REQ_STATE = {0: "queued", 1: "active", 2: "done", 3: "rejected", 4: "cancelled"}

_dp = ctypes.POINTER(ctypes.c_double)
_szp = ctypes.POINTER(ctypes.c_size_t)
_vp = ctypes.c_void_p


class PawanError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class ServeConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_double), ("max_step_interactions", ctypes.c_double),
                ("max_active", ctypes.c_int), ("max_queue", ctypes.c_int),
                ("precision", ctypes.c_int), ("iteration_seconds", ctypes.c_double),
                ("policy", ctypes.c_int)]


class Tiling(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("threads_per_target", ctypes.c_int),
                ("targets_per_thread", ctypes.c_int), ("unroll", ctypes.c_int),
                ("blocks_per_sm", ctypes.c_int), ("items_per_slot", ctypes.c_int), ("packed", ctypes.c_int),
                ("split_near", ctypes.c_int)]


def _tiling(threads, threads_per_target=1, unroll=4, items_per_slot=16, targets_per_thread=1,
            blocks_per_sm=0, packed=0, split_near=0) -> Tiling:
    """packed: 0 one source per instruction on far tiles; 1 two sources per FP32x2
    instruction with 1/rho^2 from the MUFU reciprocal; 2 the same with 1/rho^2
    from rsqrt squared (True means 1)."""
    return Tiling(threads, threads_per_target, targets_per_thread, unroll, blocks_per_sm, items_per_slot,
                  int(packed), int(split_near))


class ServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_ulonglong), ("admitted", ctypes.c_ulonglong),
                ("completed", ctypes.c_ulonglong), ("rejected", ctypes.c_ulonglong),
                ("queued", ctypes.c_ulonglong), ("active", ctypes.c_ulonglong),
                ("iterations", ctypes.c_ulonglong), ("interactions", ctypes.c_double),
                ("busy_seconds", ctypes.c_double), ("bytes_in_use", ctypes.c_double),
                ("admit_seconds", ctypes.c_double), ("plan_seconds", ctypes.c_double),
                ("retire_seconds", ctypes.c_double)]


# name -> (restype, argtypes)
_SIGS = {
    "pawan_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "pawan_ctx_destroy": (None, [_vp]),
    "pawan_ctx_last_error": (ctypes.c_char_p, [_vp]),
    "pawan_status_name": (ctypes.c_char_p, [ctypes.c_int]),
    "pawan_ctx_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int), _szp]),
    "pawan_ctx_synchronize": (ctypes.c_int, [_vp]),
    "pawan_ctx_launch_count": (ctypes.c_ulonglong, [_vp]),
    "pawan_ctx_profile": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pawan_ctx_profile_read": (ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_ulonglong), _dp]),
    "pawan_ctx_mark": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pawan_ctx_elapsed": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp]),
    "pawan_ctx_flush_l2": (ctypes.c_int, [_vp, ctypes.c_size_t]),
    "pawan_host_alloc": (ctypes.c_int, [_vp, ctypes.c_size_t, ctypes.POINTER(_vp)]),
    "pawan_host_free": (ctypes.c_int, [_vp, _vp]),
    "pawan_system_create": (ctypes.c_int, [_vp, ctypes.c_size_t, _szp, ctypes.c_double, ctypes.c_int,
                                           ctypes.POINTER(_vp)]),
    "pawan_system_destroy": (None, [_vp]),
    "pawan_system_size": (ctypes.c_size_t, [_vp]),
    "pawan_system_num_particles": (ctypes.c_size_t, [_vp]),
    "pawan_system_set_particles": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "pawan_system_set_states": (ctypes.c_int, [_vp, _dp, ctypes.c_size_t]),
    "pawan_system_get_states": (ctypes.c_int, [_vp, _dp, ctypes.c_size_t]),
    "pawan_system_solve": (ctypes.c_int, [_vp]),
    "pawan_system_get_rates": (ctypes.c_int, [_vp, _dp, ctypes.c_size_t]),
    "pawan_system_get_wake_rates": (ctypes.c_int, [_vp, ctypes.c_size_t, _dp, _dp]),
    "pawan_system_rk4": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_size_t]),
    "pawan_system_rk4_graph": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_size_t]),
    "pawan_system_euler": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_size_t]),
    "pawan_system_diagnose": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "pawan_system_kinetic_energy": (ctypes.c_int, [_vp, _dp]),
    "pawan_system_influence": (ctypes.c_int, [_vp, _dp, ctypes.c_size_t]),
    "pawan_system_influence_columns": (ctypes.c_int, [_vp, ctypes.c_size_t, _dp, _dp, ctypes.c_size_t]),
    "pawan_shard_size": (ctypes.c_size_t, [ctypes.c_size_t, ctypes.c_int]),
    "pawan_system_set_kernel": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pawan_ctx_profile_stage": (ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_ulonglong), _dp]),
    "pawan_system_integrate": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_size_t, ctypes.c_char_p,
                                              ctypes.c_int]),
    "pawan_system_integrate_file": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_size_t, _vp, ctypes.c_int]),
    "pawan_server_inject": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "pawan_system_get_kernel": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    "pawan_system_set_shard": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "pawan_system_shard_rates": (ctypes.c_int, [_vp]),
    "pawan_system_shard_stage": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double]),
    "pawan_ctx_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "pawan_system_set_nu": (ctypes.c_int, [_vp, ctypes.c_double]),
    "pawan_system_set_precision": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pawan_system_write_frame": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_double, ctypes.c_int]),
    "pawan_system_set_tiling": (ctypes.c_int, [_vp, ctypes.POINTER(Tiling)]),
    "pawan_system_get_tiling": (ctypes.c_int, [_vp, ctypes.POINTER(Tiling)]),
    "pawan_system_autotune": (ctypes.c_int, [_vp]),
    "pawan_tile_candidates": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(Tiling), ctypes.c_size_t,
                                             _szp]),
    "pawan_tile_chunkings": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.c_size_t, _szp]),
    "pawan_system_device_state": (ctypes.c_int, [_vp, ctypes.POINTER(_dp)]),
    "pawan_system_checkpoint": (ctypes.c_int, [_vp]),
    "pawan_system_restore": (ctypes.c_int, [_vp]),
    "pawan_batch_create": (ctypes.c_int, [_vp, ctypes.c_size_t, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "pawan_batch_destroy": (None, [_vp]),
    "pawan_batch_rk4": (ctypes.c_int, [_vp, _dp, ctypes.c_double, ctypes.c_size_t, ctypes.c_int]),
    "pawan_batch_solve": (ctypes.c_int, [_vp]),
    "pawan_batch_set_tiling": (ctypes.c_int, [_vp, ctypes.POINTER(Tiling)]),
    "pawan_batch_autotune": (ctypes.c_int, [_vp]),
    "pawan_server_create": (ctypes.c_int, [_vp, ctypes.POINTER(ServeConfig), ctypes.POINTER(_vp)]),
    "pawan_server_destroy": (None, [_vp]),
    "pawan_server_submit": (ctypes.c_int, [_vp, ctypes.c_size_t, _szp, _dp, _dp, _dp, _dp, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_size_t, ctypes.POINTER(ctypes.c_longlong)]),
    "pawan_server_poll": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int)]),
    "pawan_server_wait": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_double]),
    "pawan_server_fetch": (ctypes.c_int, [_vp, ctypes.c_longlong, _dp, ctypes.c_size_t, _dp, _dp, _dp]),
    "pawan_server_cancel": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "pawan_server_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ServeStats)]),
    "pawan_server_get_tiling": (ctypes.c_int, [_vp, ctypes.POINTER(Tiling)]),
    "pawan_interact_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p]),
    "pawan_peak_fp32": (ctypes.c_int, [_vp, ctypes.c_double, _dp]),
    "pawan_peak_fp64": (ctypes.c_int, [_vp, ctypes.c_double, _dp]),
}

_lib = None


def load_library():
    """Loads the CUDA library; raises (no fallback) if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"pawan_b200 CUDA library missing: {LIB_PATH} "
                              "(build it with `python -m pawan_b200.build`)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _f64(a, shape=None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and out.shape != shape:
        out = out.reshape(shape)
    return out


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Context:
    """One device and stream (C: ``pawan_ctx``)."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        h = _vp()
        st = self._lib.pawan_ctx_create(int(device), ctypes.byref(h))
        if st != OK:
            raise PawanError(st, f"cannot create a context on CUDA device {device} "
                                 "(needs a B200 / sm_100 device)")
        self._h = h
        self.device = device
        import weakref
        self._children = weakref.WeakSet()

    def _adopt(self, child):
        self._children.add(child)

    @property
    def stream(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        s = _vp()
        self.check(self._lib.pawan_ctx_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    @property
    def handle(self):
        return self._h

    def check(self, st: int):
        if st != OK:
            msg = self._lib.pawan_ctx_last_error(self._h)
            raise PawanError(st, msg.decode() if msg else "")

    def close(self):
        """Destroys the context, after the systems, batches and servers made on it."""
        if getattr(self, "_h", None):
            for child in list(getattr(self, "_children", ())):
                child.close()
            self._lib.pawan_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def info(self) -> dict:
        sm, ma, mi, mem = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        self.check(self._lib.pawan_ctx_info(self._h, ctypes.byref(sm), ctypes.byref(ma), ctypes.byref(mi),
                                            ctypes.byref(mem)))
        return {"sm_count": sm.value, "cc": (ma.value, mi.value), "total_mem": mem.value}

    def synchronize(self):
        self.check(self._lib.pawan_ctx_synchronize(self._h))

    @property
    def launch_count(self) -> int:
        return int(self._lib.pawan_ctx_launch_count(self._h))

    def profile(self, enable: bool = True):
        self.check(self._lib.pawan_ctx_profile(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        ms, n, inter = ctypes.c_double(), ctypes.c_ulonglong(), ctypes.c_double()
        self.check(self._lib.pawan_ctx_profile_read(self._h, ctypes.byref(ms), ctypes.byref(n),
                                                    ctypes.byref(inter)))
        return {"pair_ms": ms.value, "pair_launches": n.value, "pair_interactions": inter.value}

    def profile_stage(self) -> dict:
        """Stage-kernel totals since profiling was enabled: ms, launches, and
        algorithmic HBM bytes."""
        ms, n, b = ctypes.c_double(), ctypes.c_ulonglong(), ctypes.c_double()
        self.check(self._lib.pawan_ctx_profile_stage(self._h, ctypes.byref(ms), ctypes.byref(n),
                                                     ctypes.byref(b)))
        return {"stage_ms": ms.value, "stage_launches": n.value, "stage_bytes": b.value}

    def mark(self, slot: int):
        self.check(self._lib.pawan_ctx_mark(self._h, int(slot)))

    def elapsed_ms(self, slot0: int, slot1: int) -> float:
        v = ctypes.c_double()
        self.check(self._lib.pawan_ctx_elapsed(self._h, int(slot0), int(slot1), ctypes.byref(v)))
        return v.value

    def flush_l2(self, nbytes: int = 256 << 20):
        self.check(self._lib.pawan_ctx_flush_l2(self._h, int(nbytes)))

    def pinned(self, shape, dtype=np.float64) -> np.ndarray:
        """A numpy array in pinned (page-locked) host memory, freed with the array."""
        nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        ptr = _vp()
        self.check(self._lib.pawan_host_alloc(self._h, nbytes, ctypes.byref(ptr)))
        buf = (ctypes.c_char * max(1, nbytes)).from_address(ptr.value)
        arr = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)
        lib, h, p = self._lib, self._h, ptr.value
        import weakref
        weakref.finalize(buf, lambda: lib.pawan_host_free(h, ctypes.c_void_p(p)))
        return arr

    def peak_fp32(self, seconds: float = 1.0) -> float:
        g = ctypes.c_double()
        self.check(self._lib.pawan_peak_fp32(self._h, float(seconds), ctypes.byref(g)))
        return g.value

    def peak_fp64(self, seconds: float = 1.0) -> float:
        g = ctypes.c_double()
        self.check(self._lib.pawan_peak_fp64(self._h, float(seconds), ctypes.byref(g)))
        return g.value


class System:
    """``pawan::__interaction`` over its wakes, on the GPU (C: ``pawan_system``)."""

    def __init__(self, ctx: Context, counts: Sequence[int], nu: float, precision: str = "f32"):
        self.ctx = ctx
        self._lib = ctx._lib
        self.counts = [int(c) for c in counts]
        cnt = np.asarray(self.counts, dtype=np.uintp)
        h = _vp()
        ctx.check(self._lib.pawan_system_create(ctx.handle, len(self.counts), cnt.ctypes.data_as(_szp),
                                                float(nu), PREC[precision], ctypes.byref(h)))
        self._h = h
        ctx._adopt(self)
        self.n = sum(self.counts)
        self.size = 6 * self.n
        self.nu = nu
        self.precision = precision

    @classmethod
    def from_scenario(cls, ctx: Context, sc, precision: str = "f32") -> "System":
        s = cls(ctx, sc.counts, sc.nu, precision)
        s.set_particles(*sc.union())
        return s

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pawan_system_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_particles(self, pos, vor, rad, vol):
        pos, vor = _f64(pos, (self.n, 3)), _f64(vor, (self.n, 3))
        rad, vol = _f64(rad, (self.n,)), _f64(vol, (self.n,))
        self.ctx.check(self._lib.pawan_system_set_particles(self._h, _p(pos), _p(vor), _p(rad), _p(vol)))

    def set_states(self, state):
        s = _f64(state, (self.size,))
        self.ctx.check(self._lib.pawan_system_set_states(self._h, _p(s), self.size))

    def get_states(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        s = np.empty(self.size) if out is None else out
        self.ctx.check(self._lib.pawan_system_get_states(self._h, _p(s), self.size))
        return s

    def solve(self):
        self.ctx.check(self._lib.pawan_system_solve(self._h))

    def get_rates(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        r = np.empty(self.size) if out is None else out
        self.ctx.check(self._lib.pawan_system_get_rates(self._h, _p(r), self.size))
        return r

    def wake_rates(self, w: int):
        c = self.counts[w]
        u, da = np.empty((c, 3)), np.empty((c, 3))
        self.ctx.check(self._lib.pawan_system_get_wake_rates(self._h, w, _p(u), _p(da)))
        return u, da

    def union_rates(self):
        us, das = zip(*(self.wake_rates(w) for w in range(len(self.counts))))
        return np.concatenate(us), np.concatenate(das)

    def rk4(self, dt: float, nsteps: int = 1, use_graph: bool = False):
        """nsteps of __rk4::step on the device; use_graph replays the step's
        launches from a CUDA graph (same bits)."""
        fn = self._lib.pawan_system_rk4_graph if use_graph else self._lib.pawan_system_rk4
        self.ctx.check(fn(self._h, float(dt), int(nsteps)))

    def euler(self, dt: float, nsteps: int = 1):
        self.ctx.check(self._lib.pawan_system_euler(self._h, float(dt), int(nsteps)))

    def diagnose(self, quadratic: bool = True) -> dict:
        out = np.zeros(11)
        self.ctx.check(self._lib.pawan_system_diagnose(self._h, _p(out), 1 if quadratic else 0))
        return {"total_vorticity": out[0:3].copy(), "linear_impulse": out[3:6].copy(),
                "angular_impulse": out[6:9].copy(), "enstrophy": float(out[9]),
                "helicity": float(out[10])}

    def kinetic_energy(self) -> float:
        v = ctypes.c_double()
        self.ctx.check(self._lib.pawan_system_kinetic_energy(self._h, ctypes.byref(v)))
        return v.value

    def integrate(self, T: float, n: int, path: str, method: str = "rk4"):
        """The reference's integrate(): n steps of T/n with a .wake frame at t = 0
        and after every step, written to `path` asynchronously."""
        m = {"rk4": 0, "euler": 1}[method]
        self.ctx.check(self._lib.pawan_system_integrate(self._h, float(T), int(n), os.fsencode(path), m))

    def set_kernel(self, kernel: str):
        """Smoothing kernel: "highorder" (the reference's default) or "gaussian"."""
        self.ctx.check(self._lib.pawan_system_set_kernel(self._h, KERNELS[kernel]))

    @property
    def kernel(self) -> str:
        k = ctypes.c_int()
        self.ctx.check(self._lib.pawan_system_get_kernel(self._h, ctypes.byref(k)))
        return {v: n for n, v in KERNELS.items()}[k.value]

    def influence(self) -> np.ndarray:
        """Vorticity field of every particle (N x 3, FP64): the reference's
        ``__interaction::resolve()`` / ``influence()``."""
        k = np.empty((self.n, 3))
        self.ctx.check(self._lib.pawan_system_influence(self._h, _p(k), k.size))
        return k

    def influence_columns(self, alpha) -> np.ndarray:
        """Vorticity field of several strength vectors over the current
        positions and radii: ``alpha`` is (C, N, 3), the result (C, N, 3).
        The influence-matrix columns of ``__resolve::rebuild``, one launch per
        group of columns; the system's own strengths are unchanged."""
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        if a.ndim != 3 or a.shape[1:] != (self.n, 3):
            raise ValueError(f"alpha must be (C, {self.n}, 3)")
        k = np.empty_like(a)
        self.ctx.check(self._lib.pawan_system_influence_columns(self._h, a.shape[0], _p(a), _p(k),
                                                                 k.size))
        return k

    def set_nu(self, nu: float):
        self.ctx.check(self._lib.pawan_system_set_nu(self._h, float(nu)))
        self.nu = nu

    def set_precision(self, precision: str):
        self.ctx.check(self._lib.pawan_system_set_precision(self._h, PREC[precision]))
        self.precision = precision

    def write_frame(self, path: str, t: float, append: bool = True):
        self.ctx.check(self._lib.pawan_system_write_frame(self._h, os.fsencode(path), float(t),
                                                          1 if append else 0))

    def set_config(self, threads: int, threads_per_target: int = 1, unroll: int = 4,
                   items_per_slot: int = 16, targets_per_thread: int = 1, blocks_per_sm: int = 0,
                   packed: int = 0, split_near: int = 0):
        t = _tiling(threads, threads_per_target, unroll, items_per_slot, targets_per_thread, blocks_per_sm,
                    packed, split_near)
        self.ctx.check(self._lib.pawan_system_set_tiling(self._h, ctypes.byref(t)))

    def get_config(self) -> dict:
        t = Tiling()
        self.ctx.check(self._lib.pawan_system_get_tiling(self._h, ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in Tiling._fields_}

    def autotune(self) -> dict:
        self.ctx.check(self._lib.pawan_system_autotune(self._h))
        return self.get_config()

    def checkpoint(self):
        """Device-side snapshot of the state."""
        self.ctx.check(self._lib.pawan_system_checkpoint(self._h))

    def restore(self):
        """Back to the last checkpoint (device to device)."""
        self.ctx.check(self._lib.pawan_system_restore(self._h))


class Batch:
    """Independent systems in one persistent launch per RK4 stage (C: ``pawan_batch``)."""

    def __init__(self, ctx: Context, systems: Sequence[System]):
        self.ctx = ctx
        self._lib = ctx._lib
        self.systems = list(systems)
        arr = (_vp * len(self.systems))(*[s.handle for s in self.systems])
        h = _vp()
        ctx.check(self._lib.pawan_batch_create(ctx.handle, len(self.systems), arr, ctypes.byref(h)))
        self._h = h
        ctx._adopt(self)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pawan_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rk4(self, dt, nsteps: int = 1, use_graph: bool = True):
        if np.isscalar(dt):
            self.ctx.check(self._lib.pawan_batch_rk4(self._h, None, float(dt), int(nsteps), int(use_graph)))
        else:
            d = _f64(dt, (len(self.systems),))
            self.ctx.check(self._lib.pawan_batch_rk4(self._h, _p(d), 0.0, int(nsteps), int(use_graph)))

    def solve(self):
        self.ctx.check(self._lib.pawan_batch_solve(self._h))

    def set_config(self, threads: int, threads_per_target: int = 1, unroll: int = 4,
                   items_per_slot: int = 16, targets_per_thread: int = 1, blocks_per_sm: int = 0,
                   packed: int = 0, split_near: int = 0):
        t = _tiling(threads, threads_per_target, unroll, items_per_slot, targets_per_thread, blocks_per_sm,
                    packed, split_near)
        self.ctx.check(self._lib.pawan_batch_set_tiling(self._h, ctypes.byref(t)))

    def autotune(self):
        self.ctx.check(self._lib.pawan_batch_autotune(self._h))


class Server:
    """Continuous-batching request loop (C: ``pawan_server``)."""

    def __init__(self, ctx: Context, budget_bytes: float, max_step_interactions: float = 0.0,
                 max_active: int = 0, max_queue: int = 0, precision: str = "f32",
                 iteration_seconds: float = 0.0, policy: str = "fifo"):
        """iteration_seconds: device time one engine iteration may take before
        new arrivals are admitted (0: the engine's default of 20 ms; a tiny value
        gives one RK4 step per iteration).  policy: "fifo" (arrival order) or
        "shortest" (least N^2 x steps first)."""
        self.ctx = ctx
        self._lib = ctx._lib
        cfg = ServeConfig(float(budget_bytes), float(max_step_interactions), int(max_active),
                          int(max_queue), PREC[precision], float(iteration_seconds),
                          {"fifo": 0, "shortest": 1}[policy])
        h = _vp()
        ctx.check(self._lib.pawan_server_create(ctx.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._sizes = {}
        ctx._adopt(self)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pawan_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, counts, pos, vor, rad, vol, nu: float, dt: float, nsteps: int) -> tuple:
        """Returns (status, id); status != 0 means rejected at submission."""
        counts = [int(c) for c in counts]
        n = sum(counts)
        cnt = np.asarray(counts, dtype=np.uintp)
        pos, vor = _f64(pos, (n, 3)), _f64(vor, (n, 3))
        rad, vol = _f64(rad, (n,)), _f64(vol, (n,))
        rid = ctypes.c_longlong()
        st = self._lib.pawan_server_submit(self._h, len(counts), cnt.ctypes.data_as(_szp), _p(pos), _p(vor),
                                           _p(rad), _p(vol), float(nu), float(dt), int(nsteps),
                                           ctypes.byref(rid))
        self._sizes[rid.value] = 6 * n
        return st, rid.value

    def submit_scenario(self, sc, nsteps: Optional[int] = None) -> tuple:
        return self.submit(sc.counts, *sc.union(), sc.nu, sc.dt, sc.steps if nsteps is None else nsteps)

    def poll(self, rid: int) -> str:
        s = ctypes.c_int()
        st = self._lib.pawan_server_poll(self._h, rid, ctypes.byref(s))
        if st != OK:
            raise PawanError(st, f"request {rid}")
        return REQ_STATE[s.value]

    def wait(self, rid: int, timeout: float = 60.0) -> bool:
        st = self._lib.pawan_server_wait(self._h, rid, float(timeout))
        if st == 6:
            return False
        if st != OK:
            raise PawanError(st, f"request {rid}")
        return True

    def fetch(self, rid: int):
        """(state or None, t_submit, t_admit, t_done) of a finished request."""
        size = self._sizes.get(rid, 0)
        out = np.empty(size)
        ts, ta, td = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        st = self._lib.pawan_server_fetch(self._h, rid, _p(out), size, ctypes.byref(ts), ctypes.byref(ta),
                                          ctypes.byref(td))
        if st not in (OK, 4, 8):
            raise PawanError(st, f"request {rid}")
        self._sizes.pop(rid, None)
        return (out if st == OK else None), ts.value, ta.value, td.value

    def cancel(self, rid: int):
        st = self._lib.pawan_server_cancel(self._h, rid)
        if st != OK:
            raise PawanError(st, f"request {rid}")

    FAULTS = {"alloc": 1, "iteration": 2, "slow": 3}

    def inject(self, fault: str, count: int = 1, seconds: float = 0.0):
        """Host-side fault injection: "alloc" (admission allocation fails),
        "iteration" (an engine iteration fails), "slow" (iterations sleep
        `seconds` first)."""
        st = self._lib.pawan_server_inject(self._h, self.FAULTS[fault], int(count), float(seconds))
        if st != OK:
            raise PawanError(st, "inject")

    def stats(self) -> dict:
        s = ServeStats()
        st = self._lib.pawan_server_stats(self._h, ctypes.byref(s))
        if st != OK:
            raise PawanError(st, "stats")
        return {f: getattr(s, f) for f, _ in ServeStats._fields_}

    def tiling(self) -> dict:
        """The tiling of the engine's pair launches (System.set_config
        keywords), to run a request alone with the same arithmetic."""
        t = Tiling()
        st = self._lib.pawan_server_get_tiling(self._h, ctypes.byref(t))
        if st != OK:
            raise PawanError(st, "tiling")
        return {f: getattr(t, f) for f, _ in Tiling._fields_}


NOALLOC_MAX_PARTICLES = 16384


def interact_noalloc(position: int, vorticity: int, radius: int, volume: int, n: int, nu: float,
                     velocity: int, retvorcity: int, stream: int = 0) -> int:
    """The allocation-free solve on caller-owned device arrays (addresses as
    ints: n x 3 / n float64 inputs, n x 3 float64 outputs).  Returns the C
    status (0 = ok); asynchronous on `stream` (0: default stream)."""
    lib = load_library()
    return int(lib.pawan_interact_noalloc(position, vorticity, radius, volume, int(n), float(nu),
                                          velocity, retvorcity, stream or None))


def tile_candidates(precision: str = "f32", kernel: str = "highorder") -> list:
    """The tilings the autotuner times (dicts as System.get_config returns);
    host-only, no GPU needed."""
    lib = load_library()
    n = ctypes.c_size_t(0)
    st = lib.pawan_tile_candidates(PREC[precision], KERNELS[kernel], None, 0, ctypes.byref(n))
    if st != OK:
        raise PawanError(st, "tile_candidates")
    arr = (Tiling * max(1, n.value))()
    lib.pawan_tile_candidates(PREC[precision], KERNELS[kernel], arr, n.value, ctypes.byref(n))
    return [{f: getattr(arr[i], f) for f, _ in Tiling._fields_} for i in range(n.value)]


def tile_chunkings() -> list:
    """The chunkings (work items per resident block) the autotuner times."""
    lib = load_library()
    n = ctypes.c_size_t(0)
    lib.pawan_tile_chunkings(None, 0, ctypes.byref(n))
    arr = (ctypes.c_int * max(1, n.value))()
    lib.pawan_tile_chunkings(arr, n.value, ctypes.byref(n))
    return list(arr[:n.value])


def rms_rel(a, b) -> float:
    """||a - b||_2 / ||b||_2 over all components: the RMS relative error the
    tests and the bench state against a reference b."""
    a, b = np.asarray(a, dtype=np.float64).ravel(), np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def max_rel(a, b) -> float:
    """max |a - b| / max |b|: the largest error relative to the largest
    reference value (per-component relative error is ill-conditioned where
    the reference is near 0)."""
    a, b = np.asarray(a, dtype=np.float64).ravel(), np.asarray(b, dtype=np.float64).ravel()
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / den) if den > 0 else float(np.abs(a - b).max())


def error_stats(u, da, u_ref, da_ref) -> dict:
    """RMS and max relative error of velocity and vorticity rate."""
    return {"u_rms_rel": rms_rel(u, u_ref), "u_max_rel": max_rel(u, u_ref),
            "dalpha_rms_rel": rms_rel(da, da_ref), "dalpha_max_rel": max_rel(da, da_ref)}


def union_to_state(counts: Sequence[int], pos: np.ndarray, vor: np.ndarray) -> np.ndarray:
    """Union arrays -> reference state layout (per wake [x | alpha])."""
    out, o = [], 0
    for c in counts:
        out.append(pos[o:o + c].ravel())
        out.append(vor[o:o + c].ravel())
        o += c
    return np.concatenate(out)


def state_to_union(counts: Sequence[int], state: np.ndarray):
    """Reference state layout -> (pos, vor) union arrays."""
    ps, vs, o = [], [], 0
    for c in counts:
        blk = state[6 * o: 6 * (o + c)]
        ps.append(blk[:3 * c].reshape(c, 3))
        vs.append(blk[3 * c:].reshape(c, 3))
        o += c
    return np.concatenate(ps), np.concatenate(vs)
