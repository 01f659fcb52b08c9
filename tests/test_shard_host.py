"""Host side of the target sharding (pawan_b200/shard.py), on CPU: block
sizes and ownership, and the exchange layout the stage kernel reads,
all-gathered over gloo by two processes through the same gather helper the
GPU path uses with NCCL."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from pawan_b200.shard import owned_range, shard_size

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_shard_sizes_cover_every_particle_once():
    for n in (2, 511, 512, 513, 2048, 131072, 262144, 100003):
        for world in (1, 2, 3, 4, 8):
            s = shard_size(n, world)
            assert s % 512 == 0 and s * world >= n
            seen = np.zeros(n, dtype=int)
            for r in range(world):
                a, b = owned_range(n, r, world)
                assert a % 512 == 0 or a == n
                seen[a:b] += 1
            assert (seen == 1).all()
    assert shard_size(131072, 8) == 16384
    assert shard_size(10, 0) == 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _value(rank, k, i):
    return rank * 1e6 + k * 1e4 + i


def _rank_main(rank, world, port, n, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from pawan_b200.shard import owned_range, shard_size, torch_allgather
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        S = shard_size(n, world)
        send = torch.empty(6 * S, dtype=torch.float64)
        a, b = owned_range(n, rank, world)
        for k in range(6):
            for i in range(S):
                send[k * S + i] = _value(rank, k, i) if a + i < b else -1.0
        recv = torch.zeros(6 * S * world, dtype=torch.float64)
        torch_allgather()(recv, send)
        # what the stage kernel reads for particle l, component k
        ok = True
        for l in range(n):
            for k in range(6):
                got = recv[(l // S) * 6 * S + k * S + l % S].item()
                ok &= got == _value(l // S, k, l % S)
        out.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [1000, 1536])
def test_exchange_layout_over_gloo(n):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert res == [(0, True), (1, True)]
