"""Multi-rank host logic of bench.py over gloo on CPU (world size 2): rank
discovery from the torchrun environment, barriers, the max-over-ranks timing
reduction and the whole-job aggregation, and the reference arm under torchrun
(rank 0 alone runs and prints; the other ranks exit 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "PAWAN_BENCH_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    import bench
    rk = bench.Ranks(world)
    try:
        rk.barrier()
        local_ms = 100.0 + 50.0 * rank     # rank 1 is the slow one
        ms_max = rk.max(local_ms)
        rate = bench.aggregate_rate(rk.world, 4.0e9, ms_max)
        rk.barrier()
        out.put((rank, rk.world, ms_max, rate))
    finally:
        rk.close()


def test_two_ranks_take_the_max_and_aggregate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, w, ms_max, rate in res:
        assert w == 2 and ms_max == 150.0
        assert rate == pytest.approx(2 * 4.0e9 / 0.150 / 1e9)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    rk = bench.Ranks(1)
    assert rk.world == 1 and rk.dist is None and rk.max(3.5) == 3.5
    rk.close()


def test_reference_arm_under_two_ranks():
    sys.path.insert(0, ROOT)
    import oracle
    if not oracle.ref_available():
        pytest.skip("the reference's sources are not compiled here (make -C oracle)")
    env = dict(os.environ, PAWAN_BENCH_BACKEND="gloo", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "1", "--n-stations", "128"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["config"]["n_particles"] == 2048
