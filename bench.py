#!/usr/bin/env python
"""Headline benchmark: all-pairs vortex-particle interaction driven by RK4.

Workload: the leapfrogging coaxial ring pair, N = 131,072 (2 wakes x 8,192
stations x 8 core particles), nu = 1e-4 with PSE diffusion, dt = 0.005; FP32
pair math with FP64 accumulation, FP64 RK4 state.  One step = one RK4 step =
4 right-hand sides = 4 N^2 pair interactions (the N-body convention; the
reference's symmetric loop evaluates N(N-1)/2 kernels per RHS for the same
credit).  Seeded synthetic geometry (no dataset exists for this path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pawan|reference] [--strong]

Prints one JSON line (rank 0).  `value` is device-timed throughput with the
state resident in HBM; `e2e` is the same metric through the C ABI with host
buffers (state H2D and D2H every step); `roofline` is the FP32 pair kernel's
algorithmic flop rate (96 flops per interaction with diffusion) against the
FP32 FFMA throughput measured in the same run; `state_update` is the
per-particle RK4 stage kernel's algorithmic HBM bytes per launch over its
CUDA-event time, against the measured copy bandwidth; `cpu_baseline` is the
reference's own OpenMP __parallel::solve (compiled from its sources) on a
bounded sample, on this host's cores.  With --gpus N (torchrun), every rank
runs its own ring pair (independent replicas, weak scaling); the time is the
max over ranks.  With --strong the ranks instead share ONE ring pair: each
computes the rates of its block of targets and the blocks are all-gathered
over NCCL on every RK4 stage (pawan_b200/shard.py); value is that one
system's interactions over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOPS_NU = 96      # algorithmic flops per interaction with diffusion
FLOPS_NO_NU = 79   # without (nu = 0)
METRIC = "G pair-interactions/s at N=131k vs plain FP64 GPU; batched solves/s, p99 latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["pawan", "reference"], default="pawan")
    ap.add_argument("--n-stations", type=int, default=8192, help="stations per ring (8 particles each)")
    ap.add_argument("--quick", action="store_true",
                    help="main timed loop only (no autotune, FP64 comparison, e2e, CPU baseline)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-suite", action="store_true", help="skip the batch and serving legs")
    ap.add_argument("--configs", action="store_true",
                    help="run every workload at its full length instead (minutes; one JSON line each)")
    ap.add_argument("--strong", action="store_true",
                    help="one system sharded over the ranks (all-gather per RK4 stage) instead of "
                         "one replica per rank")
    ap.add_argument("--batch-rhs", action="store_true",
                    help="profiling aid: right-hand sides of the 512-solve ragged batch only (the "
                         "autotuned tiling, or --tile), timed with CUDA events; one JSON line")
    ap.add_argument("--tile", default=None,
                    help="fixed FP32 tiling instead of the autotuned one: threads,threads_per_target,"
                         "targets_per_thread,unroll,blocks_per_sm,packed[,items_per_slot[,split_near]]")
    return ap.parse_args()


def apply_tile(s, spec: str):
    v = [int(x) for x in spec.split(",")]
    tb, p, r, unroll, minb, packed = v[:6]
    ips = v[6] if len(v) > 6 else 32
    split = v[7] if len(v) > 7 else 0
    s.set_config(tb, p, unroll, ips, targets_per_thread=r, blocks_per_sm=minb, packed=packed, split_near=split)
    return s.get_config()


# ------------------------------------------------------------------ ranks

class Ranks:
    """One process per GPU (torchrun env).  NCCL for the timing reductions; the
    multi-rank tests run the same code over gloo on CPU (PAWAN_BENCH_BACKEND)."""

    def __init__(self, gpus: int, backend: str = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or os.environ.get("PAWAN_BENCH_BACKEND", "nccl")
        self.dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            timeout = datetime.timedelta(seconds=120)
            if self.backend == "nccl":
                torch.cuda.set_device(self.local)
                dist.init_process_group("nccl", timeout=timeout,
                                        device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group(self.backend, timeout=timeout)
            self.dist = dist
            self.torch = torch

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if not self.dist:
            return v
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([v], dtype=self.torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


def aggregate_rate(world: int, interactions_per_rank: float, ms_max: float) -> float:
    """Whole-job G interactions/s: every rank's work over the slowest rank's time."""
    return world * interactions_per_rank / (ms_max * 1e-3) / 1e9


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None}


def gpu_processes(index: int) -> int:
    """Compute processes nvidia-smi lists on the GPU (other tenants slow a run)."""
    try:
        out = subprocess.run(["nvidia-smi", "-i", str(index), "--query-compute-apps=pid",
                              "--format=csv,noheader"], capture_output=True, text=True, timeout=20).stdout
        return len([l for l in out.splitlines() if l.strip()])
    except (OSError, subprocess.SubprocessError):
        return -1


def gpu_index(local: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    parts = [p for p in vis.split(",") if p.strip()]
    if parts and parts[min(local, len(parts) - 1)].strip().isdigit():
        return int(parts[min(local, len(parts) - 1)])
    return local


def profile_summary() -> dict:
    """Figures of the committed ncu summary of the pair kernel, if any."""
    p = os.path.join(ROOT, "profiles", "pair_f32_ring_pair.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except (OSError, ValueError):
            return {}
    return {}


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json, else
    the earlier measurement on these GPUs."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured: MEASURED_PEAKS.json hbm_gbs"
    except (OSError, ValueError, KeyError, TypeError):
        return 6650.0, "fallback: 6.65 TB/s measured earlier on these GPUs"


def state_update_roofline(prof_stage: dict) -> dict:
    """HBM roofline of the per-particle stage kernel (RK4 stage update and
    repack) over the timed steps: algorithmic bytes / CUDA-event time."""
    peak, src = hbm_peak()
    n = max(1, prof_stage["stage_launches"])
    ms = prof_stage["stage_ms"] / n
    gbs = prof_stage["stage_bytes"] / n / (ms * 1e-3) / 1e9 if ms > 0 else None
    return {"kernel": "stage_kernel", "bound": "hbm", "launches": prof_stage["stage_launches"],
            "ms_per_launch": ms, "bytes_per_launch": prof_stage["stage_bytes"] / n,
            "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": (gbs / peak) if gbs else None,
            "peak_source": src,
            "bytes": "per particle: the 48-byte rates the pair kernel summed, the FP64 state vectors "
                     "the stage reads and writes, radius and volume, and 128 bytes of packed tile data "
                     "(336-384 bytes for an RK4 stage)"}


def profiled_tiling_matches(tile: dict) -> bool:
    """Whether the committed ncu summary was captured with this tiling: its
    pipe and traffic figures depend on the block shape and far-path mode.  The
    chunking (items per resident block) is not compared: the chunk sums stay in
    L2 inside the launch, so the DRAM bytes do not depend on it."""
    prof = profile_summary().get("tile")
    return bool(prof) and all(tile.get(k) == v for k, v in prof.items() if k != "items_per_slot")


def traffic_from_profiles(tile: dict):
    """DRAM bytes per pair launch from the committed ncu summary, when it was
    captured with the timed tiling; else None."""
    return profile_summary().get("dram_bytes_per_launch_full_size") if profiled_tiling_matches(tile) else None


def executed_from_profiles(tile: dict) -> dict:
    """Executed-work figures of the committed ncu summary and the tiling they
    were measured with (the same as the timed one or not, as `same_tiling` says)."""
    prof = profile_summary()
    out = {k: prof.get(k) for k in ("fma_pipe_active", "fma_pipe_lane_ops_per_interaction",
                                    "thread_instructions_per_interaction")}
    out["profiled_kernel"] = prof.get("kernel")
    out["same_tiling"] = profiled_tiling_matches(tile)
    return out


# ------------------------------------------------------------ CPU baseline

def cpu_model() -> str:
    """The host CPU's model name (as lscpu reports it), from /proc/cpuinfo."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.lower().startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_reference_sample(pos, vor, rad, vol, nu, target_s: float, cap_n: int = 16384):
    """Times the reference's OpenMP __parallel::solve() on the first n particles
    of the workload, growing n until one solve takes about target_s seconds
    (at most cap_n and the workload's own size).
    Returns (interactions per second, n, seconds, threads)."""
    import oracle
    threads = oracle.ref_max_threads()
    cap_n = min(cap_n, len(rad))
    n = min(1024, cap_n)
    while True:
        ref = oracle.RefSystem([n], pos[:n], vor[:n], rad[:n], vol[:n], nu, parallel=True)
        t0 = oracle.ref_wtime()
        ref.solve()
        dt = oracle.ref_wtime() - t0
        ref.close()
        if dt >= target_s or n >= cap_n:
            return n * n / dt, n, dt, threads
        grow = max(1.25, min(2.0, (target_s / max(dt, 1e-3)) ** 0.5))
        n = min(cap_n, int(n * grow) // 8 * 8)


def workload_name(sc) -> str:
    """The workload both arms of the bench report in config.workload."""
    return f"leapfrogging coaxial ring pair, N={sc.n}, nu={sc.nu}, dt={sc.dt}, RK4 step"


def run_reference(args, rk: Ranks):
    from pawan_b200 import geometry as g
    if rk.rank != 0:
        return
    sc = g.ring_pair(n_stations=args.n_stations, steps=1)
    pos, vor, rad, vol = sc.union()
    per_step = max(1.0, min(5.0, 150.0 / max(1, args.steps + args.warmup)))
    rate, n, dt, threads = cpu_reference_sample(pos, vor, rad, vol, sc.nu, per_step)
    import oracle
    for _ in range(args.warmup):
        ref = oracle.RefSystem([n], pos[:n], vor[:n], rad[:n], vol[:n], sc.nu, parallel=True)
        ref.solve()
        ref.close()
    times = []
    for _ in range(args.steps):
        ref = oracle.RefSystem([n], pos[:n], vor[:n], rad[:n], vol[:n], sc.nu, parallel=True)
        t0 = oracle.ref_wtime()
        ref.solve()
        times.append(oracle.ref_wtime() - t0)
        ref.close()
    tot = sum(times)
    value = args.steps * n * n / tot / 1e9
    sample = (f"one __parallel::solve() (reference OpenMP path, compiled from its sources) per step "
              f"on the first {n} particles of the ring pair; {threads} threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "G interactions/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ring pair geometry)",
            "config": {"workload": workload_name(sc), "n_particles": sc.n, "wakes": len(sc.counts),
                       "precision": "fp64 (the reference's)", "parallelism": f"host threads x{threads}",
                       "sample_particles": n},
            "cpu_baseline": {"value": value, "unit": "G interactions/s", "cores": threads,
                             "cpu_model": cpu_model(), "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "G interactions/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------- ragged batch leg

def _increment_errors(finals, refs, initials) -> dict:
    """Per-solve RMS / max relative error of the state increment (final state
    minus initial state, the part the solve computes) against a reference
    run's: worst, 90th percentile and median over the solves, and how many
    exceed the RHS tolerance (1e-5 RMS)."""
    from pawan_b200 import max_rel, rms_rel
    finite = [bool(np.all(np.isfinite(f)) and np.all(np.isfinite(r))) for f, r in zip(finals, refs)]
    pairs = [(f, r, x0) for f, r, x0, ok in zip(finals, refs, initials, finite) if ok]
    out = {"solves": len(finals), "non_finite": len(finals) - len(pairs)}
    if not pairs:
        return out
    rms = np.array([rms_rel(f - x0, r - x0) for f, r, x0 in pairs])
    mx = [max_rel(f - x0, r - x0) for f, r, x0 in pairs]
    out.update({"rms_rel_max": float(rms.max()), "rms_rel_p90": float(np.percentile(rms, 90)),
                "rms_rel_median": float(np.median(rms)), "max_rel_max": max(mx),
                "solves_above_1e-5": int((rms > 1e-5).sum())})
    return out


def _rhs_errors(rates, refs) -> dict:
    """Per-solve RMS / max relative error of one right-hand side (u, dalpha)
    against reference rates at the same state: worst and median."""
    from pawan_b200 import error_stats
    st = [error_stats(u, da, ur, dr) for (u, da), (ur, dr) in zip(rates, refs)]
    out = {"solves": len(st)}
    for k in ("u_rms_rel", "dalpha_rms_rel", "u_max_rel", "dalpha_max_rel"):
        v = [x[k] for x in st]
        out[k + "_worst"] = max(v)
        if k.endswith("rms_rel"):
            out[k + "_median"] = float(np.median(v))
    return out


TRAJECTORY_NOTE = ("state increments after several RK4 steps: the reference's singular kernel "
                   "(q ~ 1/rho^3 inside the smoothing radius) makes some of these rings diverge within "
                   "a few steps, and there any two roundings -- FP64 sums grouped differently included -- "
                   "separate; the right-hand-side errors are the arithmetic's accuracy")


def run_batch_leg(ctx, n_solves: int = 512, steps: int = 4, seed: int = 4, check_oracle: bool = True) -> dict:
    """512 independent single-ring solves (N log-uniform in [512, 16384]):
    `steps` RK4 steps of every solve as one batch (one persistent pair launch
    per stage, the step captured in a CUDA graph, tiles autotuned), against the
    same steps run one solve per launch sequence -- each solve with its own
    plan, the tiling autotuned per size class (half an octave of N) and its
    step replayed from a CUDA graph, so the ratio measures batching alone --
    and, for reference, one solve per launch with the library's default tiling
    and no graph.  solves/s = solves x (steps / 100) per second, a solve being
    the workload's 100 steps.  Accuracy: one right-hand side at the initial
    states, batched against one solve per launch (every solve), against the
    FP64 path on the GPU (16 solves spread over N) and against the FP64 oracle
    on the CPU (the 8 smallest, with check_oracle); then the same comparisons
    of the states after the 1 + steps steps."""
    from pawan_b200 import Batch, System
    from pawan_b200 import geometry as g
    scs = g.ragged_batch(n_solves=n_solves, seed=seed)
    inter = sum(4.0 * sc.n * sc.n for sc in scs) * steps
    dt = scs[0].dt
    initials = [sc.state() for sc in scs]
    batched = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    b = Batch(ctx, batched)
    b.autotune()
    b.solve()                         # one right-hand side at the initial states
    rates_b = [x.union_rates() for x in batched]
    b.rk4(dt, 1, use_graph=True)      # capture + warm-up
    ctx.synchronize()
    ctx.mark(2)
    b.rk4(dt, steps, use_graph=True)
    ctx.mark(3)
    t_b = ctx.elapsed_ms(2, 3) * 1e-3
    finals_b = [x.get_states() for x in batched]
    b.close()
    for x in batched:
        x.close()

    rates_s = []

    def one_per_launch(tuned: bool):
        solo = [System.from_scenario(ctx, sc, "f32") for sc in scs]
        if tuned:
            by_class = {}
            for x, sc in zip(solo, scs):
                key = int(2 * np.log2(sc.n))
                if key in by_class:
                    x.set_config(**by_class[key])
                else:
                    by_class[key] = x.autotune()
                x.solve()
                rates_s.append(x.union_rates())
        for x in solo:
            x.rk4(dt, 1, use_graph=tuned)   # plan (+ capture) and warm-up
        ctx.synchronize()
        ctx.mark(2)
        for x in solo:
            x.rk4(dt, steps, use_graph=tuned)
        ctx.mark(3)
        t = ctx.elapsed_ms(2, 3) * 1e-3
        finals = [x.get_states() for x in solo]
        for x in solo:
            x.close()
        return t, finals

    t_s, finals_s = one_per_launch(True)
    t_u, _ = one_per_launch(False)

    order = np.argsort([sc.n for sc in scs])
    sample = [int(order[k]) for k in np.linspace(0, len(scs) - 1, 16).astype(int)]
    small = [int(i) for i in order[:8]]
    rates64, f64 = [], []
    for i in sample:
        x = System.from_scenario(ctx, scs[i], "f64")
        x.solve()
        rates64.append(x.union_rates())
        x.rk4(dt, 1 + steps)
        f64.append(x.get_states())
        x.close()
    acc = {"rhs_vs_one_solve_per_launch": _rhs_errors(rates_b, rates_s),
           "rhs_vs_fp64_gpu_sample": dict(_rhs_errors([rates_b[i] for i in sample], rates64),
                                          N=[scs[i].n for i in sample])}
    traj = {"vs_one_solve_per_launch": _increment_errors(finals_b, finals_s, initials),
            "vs_fp64_gpu_sample": _increment_errors([finals_b[i] for i in sample], f64,
                                                    [initials[i] for i in sample])}
    if check_oracle:
        try:
            import oracle
            from pawan_b200 import union_to_state
            rates_or, refs = [], []
            for i in small:
                pos, vor, rad, vol = scs[i].union()
                rates_or.append(oracle.pairs(pos, vor, rad, vol, scs[i].nu))
                p1, v1 = oracle.rk4_step(pos, vor, rad, vol, scs[i].nu, dt, 1 + steps)
                refs.append(union_to_state(scs[i].counts, p1, v1))
            acc["rhs_vs_fp64_oracle_sample"] = dict(_rhs_errors([rates_b[i] for i in small], rates_or),
                                                    N=[scs[i].n for i in small])
            traj["vs_fp64_oracle_sample"] = _increment_errors([finals_b[i] for i in small], refs,
                                                              [initials[i] for i in small])
        except (OSError, ImportError) as e:
            acc["rhs_vs_fp64_oracle_sample"] = f"unavailable: {e}"
    acc["tolerance"] = {"rms_rel": 1e-5, "max_rel": 1e-4}
    acc["trajectory_after_steps"] = dict(traj, steps=1 + steps, note=TRAJECTORY_NOTE)

    frac = steps / 100.0
    return {"solves": n_solves, "steps_timed": steps,
            "batched": {"solves_per_s": n_solves * frac / t_b, "G_interactions_per_s": inter / t_b / 1e9,
                        "seconds": t_b},
            "one_solve_per_launch": {"solves_per_s": n_solves * frac / t_s,
                                     "G_interactions_per_s": inter / t_s / 1e9, "seconds": t_s,
                                     "how": "own plan per solve, tiling autotuned per half-octave of N, "
                                            "RK4 step replayed from a CUDA graph"},
            "one_solve_per_launch_default_tiling_no_graph": {
                "solves_per_s": n_solves * frac / t_u, "G_interactions_per_s": inter / t_u / 1e9,
                "seconds": t_u},
            "speedup": t_s / t_b, "accuracy": acc}


# -------------------------------------------------------------- serving leg

def run_serving_leg(ctx, rate: float, duration: float, n_lo: int, n_hi: int, steps_lo: int,
                    steps_hi: int, budget: float, cap: float, max_active: int, max_queue: int,
                    drain: float, seed: int = 5, policy: str = "fifo", accuracy_sample: int = 0) -> dict:
    """Replays a Poisson arrival trace against the continuous-batching server in
    real time.  Requests are built and submitted at their arrival times; when
    the server's queue is full an arrival is rejected without building it (the
    engine would reject it the same way).  After the arrival window the run
    waits up to `drain` seconds for requests in flight.  With accuracy_sample
    = k, k completed requests (spread over the completion order) are run again
    alone after the leg -- as an FP32 system on its own and on the FP64 path --
    and their served results compared with both."""
    from pawan_b200 import Server
    from pawan_b200 import geometry as g
    reqs = g.serving_requests(rate=rate, duration=duration, seed=seed, n_lo=n_lo, n_hi=n_hi,
                              steps_lo=steps_lo, steps_hi=steps_hi, build=False)
    srv = Server(ctx, budget_bytes=budget, max_step_interactions=cap, max_active=max_active,
                 max_queue=max_queue, policy=policy)
    ids, rejected_full, rejected_engine = {}, 0, 0
    t0 = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        if max_queue and srv.stats()["queued"] >= max_queue:
            rejected_full += 1
            continue
        wakes = g.request_wakes(r.scenario.meta)
        counts = [w.n for w in wakes]
        st, rid = srv.submit(counts, np.concatenate([w.pos for w in wakes]),
                             np.concatenate([w.vor for w in wakes]), np.concatenate([w.rad for w in wakes]),
                             np.concatenate([w.vol for w in wakes]), r.scenario.nu, r.scenario.dt,
                             r.scenario.steps)
        if st != 0:
            rejected_engine += 1
        else:
            ids[rid] = r
    t_arrivals = time.perf_counter() - t0
    deadline = time.perf_counter() + drain
    lat, done_inter, finished = [], 0.0, []
    pending = dict(ids)
    first = True  # requests that finished during the arrival window count too
    while pending and (first or time.perf_counter() < deadline):
        first = False
        for rid in list(pending):
            if srv.poll(rid) in ("done", "rejected", "cancelled"):
                out, ts, ta, td = srv.fetch(rid)
                r = pending.pop(rid)
                if out is not None:
                    lat.append(td - ts)
                    done_inter += 4.0 * r.scenario.meta["N"] ** 2 * r.scenario.steps
                    if accuracy_sample:
                        finished.append((r, out))
        time.sleep(0.01)
    elapsed = time.perf_counter() - t0
    st = srv.stats()
    engine_tiling = srv.tiling()
    srv.close()
    lat.sort()
    pct = (lambda q: lat[min(len(lat) - 1, int(q * len(lat)))] if lat else None)
    accuracy = (serving_accuracy(ctx, finished, accuracy_sample, engine_tiling)
                if accuracy_sample and finished else None)
    return {"accuracy": accuracy, "policy": policy, "rate_per_s": rate, "arrival_window_s": duration, "arrivals": len(reqs),
            "N_range": [n_lo, n_hi], "steps_range": [steps_lo, steps_hi],
            "budget_bytes": budget, "max_step_interactions": cap, "max_active": max_active,
            "max_queue": max_queue, "submitted": len(ids), "completed": len(lat),
            "rejected": rejected_full + rejected_engine + int(st["rejected"]),
            "queued_at_end": int(st["queued"]), "active_at_end": int(st["active"]),
            "solves_per_s": len(lat) / elapsed, "p50_latency_s": pct(0.50), "p99_latency_s": pct(0.99),
            "G_interactions_per_s_engine": st["interactions"] / max(1e-9, st["busy_seconds"]) / 1e9,
            "engine_seconds": {"iterations": st["busy_seconds"], "admission": st["admit_seconds"],
                               "planning": st["plan_seconds"], "retirement": st["retire_seconds"]},
            "engine_iterations": int(st["iterations"]),
            "elapsed_s": elapsed, "arrival_replay_s": t_arrivals}


def serving_accuracy(ctx, finished, k: int, tiling: dict) -> dict:
    """Served results of k completed requests against the same request run
    alone (FP32, its own system and plan, with the engine's tiling) and on the
    FP64 path, plus one right-hand side of each at its initial state in FP32
    against FP64."""
    from pawan_b200 import System
    from pawan_b200 import geometry as g
    pick = [finished[i] for i in np.linspace(0, len(finished) - 1, min(k, len(finished))).astype(int)]
    served, solo32, solo64, initials, sizes, rhs32, rhs64 = [], [], [], [], [], [], []
    for r, out in pick:
        wakes = g.request_wakes(r.scenario.meta)
        counts = [w.n for w in wakes]
        pos, vor = np.concatenate([w.pos for w in wakes]), np.concatenate([w.vor for w in wakes])
        rad, vol = np.concatenate([w.rad for w in wakes]), np.concatenate([w.vol for w in wakes])
        runs = []
        for prec in ("f32", "f64"):
            x = System(ctx, counts, r.scenario.nu, prec)
            x.set_particles(pos, vor, rad, vol)
            if prec == "f32":
                x.set_config(**tiling)
            if not runs:
                initials.append(x.get_states())
            x.solve()
            (rhs32 if prec == "f32" else rhs64).append(x.union_rates())
            x.rk4(r.scenario.dt, r.scenario.steps)
            runs.append(x.get_states())
            x.close()
        served.append(out)
        solo32.append(runs[0])
        solo64.append(runs[1])
        sizes.append(int(sum(counts)))
    return {"requests": len(pick), "N": sizes,
            "served_vs_alone_fp32": dict(_increment_errors(served, solo32, initials),
                                         metric="state increment of the served result against the same "
                                                "request run alone (FP32, its own plan, the engine's "
                                                "tiling)"),
            "rhs_fp32_vs_fp64_gpu": dict(_rhs_errors(rhs32, rhs64),
                                         metric="one right-hand side at the request's initial state"),
            "trajectory_vs_fp64_gpu": dict(_increment_errors(served, solo64, initials), note=TRAJECTORY_NOTE),
            "tolerance": {"rms_rel": 1e-5, "max_rel": 1e-4}}


# --------------------------------------------------------------- GPU arm

def run_pawan(args, rk: Ranks):
    import pawan_b200
    from pawan_b200 import Context, System
    from pawan_b200 import geometry as g

    sc = g.ring_pair(n_stations=args.n_stations, steps=1)
    N = sc.n
    pos, vor, rad, vol = sc.union()
    dt = sc.dt
    flops = FLOPS_NU if sc.nu != 0 else FLOPS_NO_NU
    ctx = Context(rk.local)
    info = ctx.info()
    s = System.from_scenario(ctx, sc, "f32")
    if args.tile:
        tuned = apply_tile(s, args.tile)
    else:
        tuned = s.get_config() if args.quick else s.autotune()
    # Every step starts from the specified geometry: under the reference's
    # kernel this configuration scrambles within a few steps (the jittered near
    # field moves particles many station spacings per step), which would
    # measure a different input.  The restore is a device copy plus a repack.
    s.checkpoint()

    for _ in range(args.warmup):
        s.restore()
        s.rk4(dt, 1)
        ctx.flush_l2()
    ctx.synchronize()

    rk.barrier()
    ctx.synchronize()
    clocks = ClockSampler(gpu_index(rk.local))
    clocks.start()
    ctx.profile(True)
    launches0 = ctx.launch_count
    ms = 0.0
    ctx.mark(0)
    for _ in range(args.steps):
        # the restore (device copy + repack of the initial geometry) and the L2
        # flush (256 MiB write) sit between the step's own events
        s.restore()
        ctx.mark(2)
        s.rk4(dt, 1)
        ctx.mark(3)
        ctx.flush_l2()
        ms += ctx.elapsed_ms(2, 3)
    ctx.mark(1)
    ms_bracket = ctx.elapsed_ms(0, 1)
    ctx.synchronize()
    launches = ctx.launch_count - launches0
    prof = ctx.profile_read()
    prof_stage = ctx.profile_stage()
    ctx.profile(False)
    clk = clocks.stop()
    clk["compute_processes"] = gpu_processes(gpu_index(rk.local))
    rk.barrier()
    ms_max = rk.max(ms)
    value = aggregate_rate(rk.world, 4.0 * N * N * args.steps, ms_max)

    pair_avg_s = prof["pair_ms"] / max(1, prof["pair_launches"]) * 1e-3
    achieved_tflops = N * N * flops / pair_avg_s / 1e12
    peak_tflops = ctx.peak_fp32(2.0) / 1e3
    state = s.get_states()
    assert np.all(np.isfinite(state)), "non-finite state"

    line = {"metric": METRIC, "value": value, "unit": "G interactions/s", "n_gpus": rk.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ring pair geometry, jitter 1e-4)",
            "config": {"workload": workload_name(sc),
                       "n_particles": N, "wakes": len(sc.counts), "precision": "fp32 pairs, fp64 accumulation+state",
                       "parallelism": f"replicas x{rk.world}", "l2": "flushed between timed steps (256 MiB write)",
                       "state": "restored to the initial geometry before every step (device copy)",
                       "timing": "CUDA events around each RK4 step; the restore and the L2 flush between "
                                 "steps are outside them",
                       "ms_per_step_with_restore_and_flush": ms_bracket / args.steps,
                       "tile": tuned, "sm_count": info["sm_count"]},
            "gpu_launches": int(launches), "clocks": clk,
            "roofline": {"bound": "fp32", "achieved": achieved_tflops, "peak": peak_tflops,
                         "unit": "TFLOP/s", "frac": achieved_tflops / peak_tflops,
                         "traffic": traffic_from_profiles(tuned),
                         "kernel": "pairs_f32_kernel", "flops_per_interaction": flops,
                         "pair_launch_ms": pair_avg_s * 1e3,
                         "peak_source": "measured: FFMA-chain probe (pawan_peak_fp32) in this run",
                         "note": "achieved counts the reference formula's 96 flops per interaction; the "
                                 "kernel executes fewer (per-tile crosses; Z terms formed only where they "
                                 "are above FP32 resolution), so frac can exceed 1. Executed-work "
                                 "utilisation: ncu FMA-pipe activity in executed_ncu",
                         "executed_ncu": executed_from_profiles(tuned)},
            "state_update": state_update_roofline(prof_stage)}

    if not args.quick:
        from pawan_b200 import error_stats, max_rel, rms_rel
        # the timed tiling's results at the specified geometry: one RHS and one
        # RK4 step from the initial state
        s.restore()
        s.solve()
        u32, da32 = s.union_rates()
        x0 = sc.state()
        s.restore()
        s.rk4(dt, 1)
        step32 = s.get_states()
        # plain FP64 comparator and tuned FP64 on the same workload: one RHS each
        cmp, rates64, steps64 = {}, {}, {}
        for prec in ("f64_plain", "f64"):
            s64 = System.from_scenario(ctx, sc, prec)
            s64.solve()
            ctx.synchronize()
            ctx.profile(True)
            s64.solve()
            p64 = ctx.profile_read()
            ctx.profile(False)
            rates64[prec] = s64.union_rates()
            s64.rk4(dt, 1)
            steps64[prec] = s64.get_states()
            t = p64["pair_ms"] * 1e-3
            cmp[prec] = {"value": N * N / t / 1e9, "unit": "G interactions/s", "pair_launch_ms": t * 1e3}
            s64.close()
        f32_rate = N * N / pair_avg_s / 1e9
        line["vs_plain_fp64"] = {"fp32_pair_rate": f32_rate, "fp64_plain": cmp["f64_plain"],
                                 "fp64_tuned": cmp["f64"],
                                 "speedup_vs_plain": f32_rate / cmp["f64_plain"]["value"],
                                 "speedup_vs_tuned_fp64": f32_rate / cmp["f64"]["value"]}
        line["peak_fp64_tflops"] = ctx.peak_fp64(1.0) / 1e3
        line["accuracy"] = {
            "tiling": tuned,
            "tolerance": {"rms_rel": 1e-5, "max_rel": 1e-4},
            "rhs_vs_fp64_plain_gpu": dict(error_stats(u32, da32, *rates64["f64_plain"]), particles=N,
                                          reference="the reference formula term by term in FP64 on the "
                                                    "GPU (pairs_plain_kernel), every particle"),
            "rk4_step_increment": {
                "fp32_vs_fp64_tuned_gpu": {"rms_rel": rms_rel(step32 - x0, steps64["f64"] - x0),
                                           "max_rel": max_rel(step32 - x0, steps64["f64"] - x0)},
                "fp64_plain_vs_fp64_tuned_gpu": {
                    "rms_rel": rms_rel(steps64["f64_plain"] - x0, steps64["f64"] - x0),
                    "max_rel": max_rel(steps64["f64_plain"] - x0, steps64["f64"] - x0)},
                "note": "one RK4 step from the specified geometry; its stages evaluate the rates at "
                        "states moved by 0.5-1 dt, where the singular near field amplifies any difference "
                        "in the rates: the two FP64 kernels, whose right-hand sides agree to ~1e-13, show "
                        "the amplification"},
        }

        # end to end through the C ABI: pinned host state in, RK4 step, state out
        hin = ctx.pinned((6 * N,))
        hout = ctx.pinned((6 * N,))
        hin[:] = sc.state()
        s.set_states(hin)
        s.rk4(dt, 1)
        s.get_states(hout)
        rk.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            s.set_states(hin)
            s.rk4(dt, 1)
            s.get_states(hout)
        t_e2e = rk.max(time.perf_counter() - t0)
        line["e2e"] = {"value": rk.world * 4.0 * N * N * args.steps / t_e2e / 1e9, "unit": "G interactions/s",
                       "h2d_bytes_per_step": int(hin.nbytes), "d2h_bytes_per_step": int(hout.nbytes),
                       "path": "pawan_system_set_states (pinned host) -> pawan_system_rk4 -> pawan_system_get_states"}

        if rk.world == 1 and not args.no_suite:
            line["batched"] = run_batch_leg(ctx, check_oracle=not args.no_cpu_baseline)
            # continuous batching at a capacity-matched load (request sizes scaled
            # down so latencies are observable in seconds), against serving the
            # same trace one request at a time
            cm = dict(rate=120.0, duration=8.0, n_lo=1024, n_hi=16384, steps_lo=5, steps_hi=20,
                      budget=120e9, cap=0.0, max_queue=0, drain=60.0)
            line["served"] = {"capacity_matched": run_serving_leg(ctx, max_active=0, accuracy_sample=16, **cm),
                              "capacity_matched_one_at_a_time": run_serving_leg(ctx, max_active=1, **cm),
                              "specified_load": run_serving_leg(
                                  ctx, rate=200.0, duration=10.0, n_lo=1024, n_hi=262144, steps_lo=50,
                                  steps_hi=400, budget=120e9, cap=2e11, max_active=0, max_queue=64,
                                  drain=0.0)}
        if rk.rank == 0 and rk.world == 1 and not args.no_cpu_baseline:
            # the oracle as the checker: 4,096 sampled targets summed over all N
            # sources in FP64 on the host cores
            try:
                import oracle
                t = np.sort(np.random.default_rng(0).choice(N, 4096, replace=False))
                u_or, da_or = oracle.pairs(pos, vor, rad, vol, sc.nu, targets=t)
                line["accuracy"]["rhs_vs_fp64_oracle_sampled"] = dict(
                    error_stats(u32[t], da32[t], u_or, da_or), targets=len(t), sources=N,
                    reference="FP64 C restatement of INTERACT/KERNEL (oracle/restate.c), itself "
                              "checked against the reference's compiled sources")
                up, dp = rates64["f64_plain"]
                line["accuracy"]["fp64_plain_gpu_vs_oracle_sampled"] = error_stats(up[t], dp[t], u_or, da_or)
            except (OSError, ImportError) as e:
                line["accuracy"]["rhs_vs_fp64_oracle_sampled"] = f"unavailable: {e}"
            try:
                rate, n, tsec, threads = cpu_reference_sample(pos, vor, rad, vol, sc.nu, 10.0)
                line["cpu_baseline"] = {
                    "value": rate / 1e9, "unit": "G interactions/s", "cores": threads,
                    "cpu_model": cpu_model(), "kind": "reference",
                    "sample": f"one __parallel::solve() of the reference (OpenMP, compiled from its sources) "
                              f"on the first {n} particles of the ring pair, {tsec:.1f} s"}
            except Exception as e:  # the reference build may be absent on a fresh checkout
                line["cpu_baseline"] = {"value": None, "unit": "G interactions/s", "cores": 0,
                                        "kind": "reference", "sample": f"unavailable: {e}"}
    s.close()
    ctx.close()
    if rk.rank == 0:
        print(json.dumps(line), flush=True)


def run_strong(args, rk: Ranks):
    """One ring pair sharded over the ranks: strong scaling."""
    import torch
    from pawan_b200 import Context, System
    from pawan_b200 import geometry as g
    from pawan_b200.shard import ShardedSystem, torch_allgather
    sc = g.ring_pair(n_stations=args.n_stations, steps=1)
    N, dt = sc.n, sc.dt
    ctx = Context(rk.local)
    s = System.from_scenario(ctx, sc, "f32")
    tuned = apply_tile(s, args.tile) if args.tile else s.get_config()
    s.checkpoint()
    sh = ShardedSystem(s, rk.rank, rk.world, torch_allgather() if rk.world > 1 else None)
    for _ in range(args.warmup):
        s.restore()
        sh.rk4(dt, 1)
        ctx.flush_l2()
    ctx.synchronize()
    rk.barrier()
    ctx.synchronize()
    clocks = ClockSampler(gpu_index(rk.local))
    clocks.start()
    ctx.profile(True)
    launches0 = ctx.launch_count
    ctx.mark(0)
    for _ in range(args.steps):
        s.restore()
        sh.rk4(dt, 1)
        ctx.flush_l2()
    ctx.mark(1)
    ms = ctx.elapsed_ms(0, 1)
    ctx.synchronize()
    launches = ctx.launch_count - launches0
    prof = ctx.profile_read()
    ctx.profile(False)
    clk = clocks.stop()
    rk.barrier()
    ms_max = rk.max(ms)
    value = 4.0 * N * N * args.steps / (ms_max * 1e-3) / 1e9
    st = s.get_states()
    assert np.all(np.isfinite(st)), "non-finite state"
    pair_avg_s = prof["pair_ms"] / max(1, prof["pair_launches"]) * 1e-3
    flops = FLOPS_NU if sc.nu != 0 else FLOPS_NO_NU
    own = prof["pair_interactions"] / max(1, prof["pair_launches"])
    achieved = own * flops / pair_avg_s / 1e12
    peak = ctx.peak_fp32(2.0) / 1e3
    line = {"metric": METRIC, "value": value, "unit": "G interactions/s", "n_gpus": rk.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ring pair geometry, jitter 1e-4)",
            "config": {"workload": workload_name(sc),
                       "n_particles": N, "precision": "fp32 pairs, fp64 accumulation+state",
                       "parallelism": f"target shards x{rk.world} (NCCL all-gather of 48 B/particle per RK4 stage)",
                       "shard_particles": sh.size, "allgather_bytes_per_step": 4 * 8 * 6 * sh.size * rk.world,
                       "l2": "flushed between timed steps (256 MiB write)",
                       "state": "restored to the initial geometry before every step (device copy)",
                       "tile": tuned},
            "gpu_launches": int(launches), "clocks": clk,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None, "kernel": "pairs_f32_kernel",
                         "flops_per_interaction": flops, "pair_launch_ms": pair_avg_s * 1e3,
                         "peak_source": "measured: FFMA-chain probe (pawan_peak_fp32) in this run"}}
    sh.close()
    s.close()
    ctx.close()
    if rk.rank == 0:
        print(json.dumps(line), flush=True)


def _finite_diag(d):
    return {k: (v.tolist() if hasattr(v, "tolist") else v) for k, v in d.items()}


def run_configs(args):
    """Every workload at its specified length (one GPU; minutes)."""
    import oracle
    from pawan_b200 import Context, System, union_to_state
    from pawan_b200 import geometry as g
    ctx = Context(0)
    emit = lambda d: print(json.dumps(d), flush=True)

    # 1) single ring, N = 2,048, nu = 0, dt = 0.01, 200 steps: FP64 and FP32 on the
    #    GPU, the reference's own __rk4 + __parallel on the CPU
    sc = g.single_ring()
    out = {"config": "single_ring", "N": sc.n, "steps": sc.steps, "dt": sc.dt}
    for prec in ("f64_plain", "f32"):
        s = System.from_scenario(ctx, sc, prec)
        d0 = s.diagnose()
        ctx.synchronize()
        t0 = time.perf_counter()
        for k in range(sc.steps // 10):
            s.rk4(sc.dt, 10)
            if k == 9:
                d100 = s.diagnose()
        st = s.get_states()
        t = time.perf_counter() - t0
        out[prec] = {"seconds": t, "finite_at_end": bool(np.all(np.isfinite(st))),
                     "diag_t0": _finite_diag(d0), "diag_step100": _finite_diag(d100),
                     "G_interactions_per_s": 4.0 * sc.n ** 2 * sc.steps / t / 1e9}
        s.close()
    pos, vor, rad, vol = sc.union()
    ref = oracle.RefSystem(sc.counts, pos, vor, rad, vol, sc.nu, parallel=True)
    st = sc.state()
    t0 = oracle.ref_wtime()
    st = ref.rk4(st, sc.dt, sc.steps)
    t = oracle.ref_wtime() - t0
    out["cpu_reference"] = {"seconds": t, "threads": oracle.ref_max_threads(),
                            "finite_at_end": bool(np.all(np.isfinite(st))),
                            "G_interactions_per_s": 4.0 * sc.n ** 2 * sc.steps / t / 1e9,
                            "path": "__rk4::step on __parallel (OpenMP), compiled from the reference sources"}
    emit(out)

    # 2) ring pair, N = 131,072, nu = 1e-4, dt = 0.005, 500 steps (FP32 pairs)
    # 3) helical wake, N = 262,144, nu = 1e-3, dt = 0.002, 300 steps, FP64
    #    diagnostics every 10 steps
    for sc, every in ((g.ring_pair(), 50), (g.helical_wake(), 10)):
        s = System.from_scenario(ctx, sc, "f32")
        tile = s.autotune()
        ctx.synchronize()
        diags, t_diag = [], 0.0
        ctx.profile(True)
        t0 = time.perf_counter()
        for k in range(sc.steps // every):
            s.rk4(sc.dt, every)
            ctx.synchronize()  # the steps run asynchronously; time the diagnostics alone
            td = time.perf_counter()
            d = s.diagnose()
            t_diag += time.perf_counter() - td
            diags.append({"step": (k + 1) * every, "enstrophy": d["enstrophy"],
                          "total_vorticity": d["total_vorticity"].tolist(),
                          "linear_impulse": d["linear_impulse"].tolist()})
        st = s.get_states()
        t = time.perf_counter() - t0
        prof = ctx.profile_read()
        ctx.profile(False)
        emit({"config": sc.name, "N": sc.n, "steps": sc.steps, "dt": sc.dt, "nu": sc.nu, "tile": tile,
              "seconds": t, "diagnostics_seconds": t_diag,
              "G_interactions_per_s_incl_diagnostics": 4.0 * sc.n ** 2 * sc.steps / t / 1e9,
              "pair_kernel_G_per_s": prof["pair_interactions"] / (prof["pair_ms"] * 1e-3) / 1e9,
              "finite_at_end": bool(np.all(np.isfinite(st))), "diagnostics": diags[:3] + diags[-2:]})
        s.close()

    # 4) ragged batch, 512 solves x 100 steps
    emit({"config": "ragged_batch", **run_batch_leg(ctx, steps=100)})

    # 5) serving at the specified load (60 s of arrivals) and at a capacity-matched one
    emit({"config": "serving_specified", **run_serving_leg(
        ctx, rate=200.0, duration=60.0, n_lo=1024, n_hi=262144, steps_lo=50, steps_hi=400,
        budget=120e9, cap=2e11, max_active=0, max_queue=64, drain=30.0)})
    emit({"config": "serving_specified_shortest_first", **run_serving_leg(
        ctx, rate=200.0, duration=60.0, n_lo=1024, n_hi=262144, steps_lo=50, steps_hi=400,
        budget=120e9, cap=2e11, max_active=0, max_queue=64, drain=30.0, policy="shortest")})
    emit({"config": "serving_capacity_matched", **run_serving_leg(
        ctx, rate=120.0, duration=30.0, n_lo=1024, n_hi=16384, steps_lo=5, steps_hi=20,
        budget=120e9, cap=0.0, max_active=0, max_queue=0, drain=60.0)})
    ctx.close()


def run_batch_rhs(args):
    """Right-hand sides of the 512-solve ragged batch (one launch sequence per
    RHS over every solve), the profiling counterpart of the batched leg:
    `--warmup` untimed, then `--steps` timed with CUDA events on the library's
    stream."""
    import pawan_b200
    from pawan_b200 import Batch, System
    from pawan_b200 import geometry as g
    ctx = pawan_b200.Context(0)
    scs = g.ragged_batch()
    systems = [System.from_scenario(ctx, sc, "f32") for sc in scs]
    b = Batch(ctx, systems)
    if args.tile:
        v = [int(x) for x in args.tile.split(",")]
        tb, p, r, unroll, minb, packed = v[:6]
        ips = v[6] if len(v) > 6 else 32
        split = v[7] if len(v) > 7 else 0
        b.set_config(tb, p, unroll, ips, targets_per_thread=r, blocks_per_sm=minb, packed=packed,
                     split_near=split)
        tiling = args.tile
    else:
        b.autotune()
        tiling = "autotuned"
    for _ in range(max(1, args.warmup)):
        b.solve()
    ctx.synchronize()
    ctx.profile(True)
    for _ in range(args.steps):
        b.solve()
    ctx.synchronize()
    r = ctx.profile_read()
    ctx.profile(False)
    ms = r["pair_ms"] / max(1, r["pair_launches"])
    print(json.dumps({"workload": "ragged batch, 512 solves, one right-hand side", "tiling": tiling,
                      "solves": len(scs), "interactions_per_rhs": sum(float(sc.n) ** 2 for sc in scs),
                      "ms_per_rhs": ms, "G_interactions_per_s": r["pair_interactions"] / r["pair_ms"] / 1e6}))
    b.close()
    for x in systems:
        x.close()
    ctx.close()


def main():
    args = parse()
    if args.configs:
        run_configs(args)
        return
    if args.batch_rhs:
        run_batch_rhs(args)
        return
    rk = Ranks(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rk)
        elif args.strong:
            run_strong(args, rk)
        else:
            run_pawan(args, rk)
    finally:
        rk.close()


if __name__ == "__main__":
    main()
