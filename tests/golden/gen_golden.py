"""Generates tests/golden/*.npz from the reference itself.

Runs the reference's own C++ classes (compiled from their unmodified sources
into oracle/_ref/libpawan_ref.so by `make -C oracle`) on small seeded inputs
and stores inputs and outputs.  The fixtures pin the oracle restatement and the
GPU path on machines without the reference tree.

    python tests/golden/gen_golden.py [case ...]     (no case: all of them)

Cases (all FP64, reference layout for states/rates):
  ring64_solve       one ring, 8 stations x 8, nu = 0       __interaction::solve
  pair64_solve       coaxial pair, 2 x 32, nu = 1e-3         cross-wake pairs
  helix3_solve       three helical filaments, 3 x 16, nu=2e-3
  ring64_rk4         3 x __rk4::step, dt = 0.01
  pair64_rk4         2 x __rk4::step, dt = 0.005, nu = 1e-3
  pair64_euler       2 x __integration::step, dt = 0.005
  pair64_diag        __interaction::diagnose + kinetic energy
  ring16_integrate   __rk4(0.02, 2).integrate -> data/temp.wake bytes
  pair64_influence   __interaction::resolve -> influence: the vorticity field
  vring1_influence   the same on the reference's __vring(1.0, 0.1, 1) (855
                     particles) with seeded layer strengths
  vring1_resolve     __resolve::rebuild on __vring(1.0, 0.1, 1): resolved strengths
  pair64_gauss       the coaxial pair with the reference's Gaussian kernel
                     (gaussian.h, compiled in by oracle/Makefile): solve, 2 RK4
                     steps, diagnose, vorticity field
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

import oracle  # noqa: E402
from pawan_b200 import geometry as g  # noqa: E402


def _inputs(sc):
    pos, vor, rad, vol = sc.union()
    return dict(counts=np.asarray(sc.counts, dtype=np.int64), pos=pos, vor=vor, rad=rad, vol=vol,
                nu=np.float64(sc.nu), state=sc.state())


def _save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print("wrote", name)


def main(only=()):
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libpawan_ref.so is not built (make -C oracle)")
    oracle.ref_set_threads(1)
    global _save
    write = _save

    def _save(name, **arrays):  # noqa: F811 - restricted to the requested cases
        if not only or name in only:
            write(name, **arrays)

    ring = g.single_ring(n_stations=8, seed=11)
    pair = g.ring_pair(n_stations=4, seed=12, nu=1e-3)
    helix = g.helical_wake(n_stations=2, seed=13, filaments=3, turns=1.0, nu=2e-3)

    for name, sc in (("ring64_solve", ring), ("pair64_solve", pair), ("helix3_solve", helix)):
        d = _inputs(sc)
        ref = oracle.RefSystem(sc.counts, d["pos"], d["vor"], d["rad"], d["vol"], sc.nu)
        ref.solve()
        _save(name, rates=ref.get_rates(), **d)

    for name, sc, dt, n, method in (("ring64_rk4", ring, 0.01, 3, "rk4"),
                                    ("pair64_rk4", pair, 0.005, 2, "rk4"),
                                    ("pair64_euler", pair, 0.005, 2, "euler")):
        d = _inputs(sc)
        ref = oracle.RefSystem(sc.counts, d["pos"], d["vor"], d["rad"], d["vol"], sc.nu)
        out = getattr(ref, method)(d["state"], dt, n)
        _save(name, final_state=out, dt=np.float64(dt), nsteps=np.int64(n), **d)

    d = _inputs(pair)
    ref = oracle.RefSystem(pair.counts, d["pos"], d["vor"], d["rad"], d["vol"], pair.nu)
    diag = ref.diagnose()
    _save("pair64_diag", total_vorticity=diag["total_vorticity"], linear_impulse=diag["linear_impulse"],
          angular_impulse=diag["angular_impulse"], enstrophy=np.float64(diag["enstrophy"]),
          helicity=np.float64(diag["helicity"]), kinetic_energy=np.float64(ref.kinetic_energy()), **d)

    small = g.single_ring(n_stations=2, seed=14)
    d = _inputs(small)
    ref = oracle.RefSystem(small.counts, d["pos"], d["vor"], d["rad"], d["vol"], 0.0)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        os.chdir(tmp)
        try:
            ref.integrate(0.02, 2)
        finally:
            os.chdir(cwd)
        raw = open(os.path.join(tmp, "data", "temp.wake"), "rb").read()
    _save("ring16_integrate", wake_bytes=np.frombuffer(raw, dtype=np.uint8), T=np.float64(0.02),
          nsteps=np.int64(2), **d)

    d = _inputs(pair)
    ref = oracle.RefSystem(pair.counts, d["pos"], d["vor"], d["rad"], d["vol"], pair.nu)
    _save("pair64_influence", field=ref.influence(), **d)

    v = oracle.RefVring(1.0, 0.1, 1)
    strengths = np.random.default_rng(15).uniform(0.5, 1.5, v.size)
    v.set_states(strengths)
    pos, vor, rad, vol = v.particles()
    _save("vring1_influence", strengths=strengths, pos=pos, vor=vor, rad=rad, vol=vol,
          counts=np.asarray([v.n], dtype=np.int64), field=v.influence())
    v.close()

    v = oracle.RefVring(1.0, 0.1, 1)
    pos, vor, rad, vol = v.particles()
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        os.chdir(tmp)
        try:
            resolved = v.resolve()
        finally:
            os.chdir(cwd)
    _save("vring1_resolve", radius=np.float64(1.0), core=np.float64(0.1), layers=np.int64(1),
          pos=pos, rad=rad, vol=vol, strengths=resolved)
    v.close()

    d = _inputs(pair)
    ref = oracle.RefSystem(pair.counts, d["pos"], d["vor"], d["rad"], d["vol"], pair.nu, kernel="gaussian")
    ref.solve()
    rates = ref.get_rates()
    diag = ref.diagnose()
    field = ref.influence()
    final = ref.rk4(d["state"], 0.005, 2)
    _save("pair64_gauss", rates=rates, final_state=final, dt=np.float64(0.005), nsteps=np.int64(2),
          total_vorticity=diag["total_vorticity"], linear_impulse=diag["linear_impulse"],
          enstrophy=np.float64(diag["enstrophy"]), helicity=np.float64(diag["helicity"]),
          field=field, **d)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
