"""One rank of a sharded RK4 run over torch.distributed / NCCL (launched by
tests/test_gpu_shard.py, or by torchrun for several GPUs).  Checks that every
rank ends with the same state as an unsharded run of the same steps on its
own GPU, within the FP64 partial-sum reordering (RMS 1e-12 of the increment)."""
import datetime
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    import torch
    import torch.distributed as dist
    from pawan_b200 import Context, System
    from pawan_b200 import geometry as g
    from pawan_b200.shard import ShardedSystem, torch_allgather
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", local))
    try:
        ctx = Context(local)
        sc = g.ring_pair(n_stations=128, seed=64, nu=1e-3)
        ref = System.from_scenario(ctx, sc, "f32")
        ref.rk4(sc.dt, 2)
        s = System.from_scenario(ctx, sc, "f32")
        sh = ShardedSystem(s, rank, world, torch_allgather())
        sh.rk4(sc.dt, 2)
        st, st_ref, st0 = s.get_states(), ref.get_states(), sc.state()
        err = np.linalg.norm((st - st0) - (st_ref - st0)) / np.linalg.norm(st_ref - st0)
        assert err < 1e-12, err
        if world == 1:
            assert np.array_equal(st, st_ref)
        sh.close()
        s.close()
        ref.close()
        ctx.close()
        print("shard ok", rank, world, err, flush=True)
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
