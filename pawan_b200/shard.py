"""Target sharding of one system over processes, one GPU each.

Every process holds the whole system.  Process ``rank`` of ``world`` computes
the pair rates of its contiguous block of targets against all sources
(``pawan_system_shard_rates``), the blocks are all-gathered over NVLink with
torch.distributed / NCCL on the library's own CUDA stream, and every process
applies the same RK4 stage update to all particles
(``pawan_system_shard_stage``), so the states stay bit-identical across
processes.  Per RK4 stage the exchange is 48 bytes per particle (the FP64
velocity and vorticity rate); the pair work per process is N^2 / world.

The reference has one process (its OpenMP loop splits the targets of each
source over threads, src/interaction/parallel.cpp:21); this is the same split
over GPUs.

Exchange layout (the contract with the stage kernel): ``recv`` holds the
blocks of all processes in rank order, each block laid out [6][S] -- u_x, u_y,
u_z, dalpha_x, dalpha_y, dalpha_z of its S particles -- so particle l's
component k is ``recv[(l // S) * 6 * S + k * S + l % S]``.
"""
from __future__ import annotations

from typing import Callable, Optional

from . import PawanError, System, load_library

Gather = Callable[["object", "object"], None]  # gather(recv, send)


def shard_size(n: int, world: int) -> int:
    """Particles per process block S (a multiple of 512) for N particles."""
    return int(load_library().pawan_shard_size(int(n), int(world)))


def owned_range(n: int, rank: int, world: int):
    """[first, last) of the targets process ``rank`` computes."""
    s = shard_size(n, world)
    first = min(n, rank * s)
    return first, min(n, first + s)


def torch_allgather(group=None) -> Gather:
    """All-gather of each process's block into ``recv`` through
    torch.distributed: ``all_gather_into_tensor`` on NCCL, the list form on
    gloo (CPU tests)."""
    import torch.distributed as dist

    def gather(recv, send):
        if dist.get_backend(group) == "nccl":
            dist.all_gather_into_tensor(recv, send, group=group)
        else:
            world = dist.get_world_size(group)
            parts = list(recv.view(world, -1).unbind(0))
            dist.all_gather(parts, send, group=group)
    return gather


class ShardedSystem:
    """One process's view of a system sharded over ``world`` processes.

    ``gather(recv, send)`` performs the all-gather; it is called inside a
    ``torch.cuda.stream`` context on the library's stream, so a torch
    collective is ordered after this process's rate kernel and before its
    stage kernel without a host synchronisation.  With world = 1 and no
    gather the block is copied on the device.
    """

    def __init__(self, system: System, rank: int, world: int, gather: Optional[Gather] = None):
        import torch
        self.system = system
        self.rank, self.world = int(rank), int(world)
        self.size = shard_size(system.n, world)
        dev = torch.device("cuda", system.ctx.device)
        self.send = torch.zeros(6 * self.size, dtype=torch.float64, device=dev)
        self.recv = torch.zeros(6 * self.size * self.world, dtype=torch.float64, device=dev)
        self.stream = torch.cuda.ExternalStream(system.ctx.stream, device=dev)
        if gather is None:
            if self.world != 1:
                raise ValueError("world > 1 needs a gather (e.g. torch_allgather())")
            gather = lambda recv, send: recv.copy_(send)  # noqa: E731
        self.gather = gather
        lib = system._lib
        system.ctx.check(lib.pawan_system_set_shard(system.handle, self.rank, self.world,
                                                     self.send.data_ptr(), self.recv.data_ptr()))
        # the buffers were written by torch on its stream: order the library after it
        torch.cuda.current_stream(dev).synchronize()

    @property
    def owned(self):
        return owned_range(self.system.n, self.rank, self.world)

    def rates(self):
        """This process's block of rates into ``send`` (library stream)."""
        self.system.ctx.check(self.system._lib.pawan_system_shard_rates(self.system.handle))

    def exchange(self):
        import torch
        with torch.cuda.stream(self.stream):
            self.gather(self.recv, self.send)

    def stage(self, stage: int, dt: float):
        self.system.ctx.check(self.system._lib.pawan_system_shard_stage(self.system.handle, int(stage),
                                                                          float(dt)))

    def rk4(self, dt: float, nsteps: int = 1):
        """nsteps RK4 steps: per stage, rates of the owned targets, all-gather,
        stage update of every particle."""
        for _ in range(int(nsteps)):
            for stage in (1, 2, 3, 4):
                self.rates()
                self.exchange()
                self.stage(stage, dt)

    def solve(self):
        """Rates of every particle (as System.solve) through one exchange."""
        self.rates()
        self.exchange()
        self.stage(0, 0.0)

    def close(self):
        """Back to an unsharded system (the exchange buffers are released)."""
        try:
            self.system.ctx.check(self.system._lib.pawan_system_set_shard(self.system.handle, 0, 0,
                                                                          None, None))
        except PawanError:
            pass
