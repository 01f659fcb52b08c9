"""Target sharding of one system over processes on the GPU.  Only one GPU is
available to the tests, so the ranks are emulated: W systems in one process,
each computing its own block of targets, their blocks exchanged by device
copies in the all-gather layout; the ranks' kernels never wait on one another.
A single-rank NCCL process group runs the torch.distributed path itself."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch

from pawan_b200 import System
from pawan_b200 import geometry as g
from pawan_b200.shard import ShardedSystem, owned_range
from helpers import TOL_F32_RMS, rms_rel

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_world_one_matches_unsharded_bit_for_bit(ctx):
    sc = g.ring_pair(n_stations=96, seed=61, nu=1e-3)  # N = 1,536
    ref = System.from_scenario(ctx, sc, "f32")
    ref.rk4(sc.dt, 3)
    s = System.from_scenario(ctx, sc, "f32")
    sh = ShardedSystem(s, 0, 1)
    sh.rk4(sc.dt, 3)
    assert np.array_equal(s.get_states(), ref.get_states())
    sh.solve()
    ref.solve()
    assert np.array_equal(s.get_rates(), ref.get_rates())


def emulated_rk4(shards, dt, nsteps):
    """The all-gather done as device copies between emulated ranks."""
    for _ in range(nsteps):
        for stage in (1, 2, 3, 4):
            for sh in shards:
                sh.rates()
            torch.cuda.synchronize()
            for sh in shards:
                for r, other in enumerate(shards):
                    S = other.size
                    sh.recv[r * 6 * S:(r + 1) * 6 * S].copy_(other.send)
            torch.cuda.synchronize()
            for sh in shards:
                sh.stage(stage, dt)


@pytest.mark.parametrize("world,prec", [(2, "f32"), (3, "f32"), (4, "f64")])
def test_emulated_ranks_agree_and_match_unsharded(ctx, world, prec):
    sc = g.ring_pair(n_stations=80, seed=62, nu=1e-3)  # N = 1,280: ragged last block
    ref = System.from_scenario(ctx, sc, prec)
    ref.rk4(sc.dt, 2)
    st_ref = ref.get_states()
    systems = [System.from_scenario(ctx, sc, prec) for _ in range(world)]
    shards = [ShardedSystem(s, r, world, gather=lambda recv, send: None) for r, s in enumerate(systems)]
    covered = sum(b - a for a, b in (sh.owned for sh in shards))
    assert covered == sc.n
    emulated_rk4(shards, sc.dt, 2)
    states = [s.get_states() for s in systems]
    for st in states[1:]:
        assert np.array_equal(st, states[0])   # every rank holds the same state
    st0 = sc.state()
    # only the chunking of the FP64 partial sums differs from the unsharded plan
    assert rms_rel(states[0] - st0, st_ref - st0) < 1e-12


def test_sharded_system_refuses_unsharded_calls(ctx):
    sc = g.single_ring(n_stations=16, seed=63)
    s = System.from_scenario(ctx, sc, "f32")
    sh = ShardedSystem(s, 0, 1)
    assert s._lib.pawan_system_solve(s.handle) == 4     # PAWAN_ERR_STATE
    assert s._lib.pawan_system_rk4(s.handle, 0.01, 1) == 4
    sh.close()
    s.solve()                                            # unsharded again


def _free_port():
    so = socket.socket()
    so.bind(("127.0.0.1", 0))
    p = so.getsockname()[1]
    so.close()
    return p


def test_nccl_single_rank_process_group():
    """torch.distributed over NCCL (one rank): the collective runs on the
    library's stream between the rate and stage kernels."""
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()), NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "shard_worker.py")], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "shard ok" in r.stdout
