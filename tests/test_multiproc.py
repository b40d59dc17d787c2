"""Replica runs on several ranks (bench.py --gpus N): each rank times its
own box and the job reports the slowest rank; here two gloo ranks on CPU
exercise that reduction and the rendezvous on 127.0.0.1."""
import os

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = torch.tensor([10.0 + 5.0 * rank], dtype=torch.float64)  # per-rank device time
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    n_per_rank, steps = 1000, 10
    value = n_per_rank * steps * world / (float(ms.item()) / 1e3)
    dist.barrier()
    if rank == 0:
        out.put((float(ms.item()), value))
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ms, value = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert ms == 15.0
    assert abs(value - 1000 * 10 * 2 / 0.015) < 1e-6 * value
