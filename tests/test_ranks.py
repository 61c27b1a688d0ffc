"""The multi-GPU path of bench.py (independent replicas, no collective on the
data path) with two gloo ranks on CPU: each rank's times are reduced with MAX,
the whole-job throughput counts every rank's grid against the slowest rank,
and the reference arm does its work on rank 0 only."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    times = [10.0 + 5.0 * rank, 20.0 - 3.0 * rank]  # rank 0: (10, 20); rank 1: (15, 17)
    ms, e2e = bench.max_over_ranks(times, torch.device("cpu"), world)
    value = bench.replica_throughput(1000, 4, world, ms)

    class Args:
        impl, size, steps, warmup, gpus = "reference", 33, 1, 0, world

    ran_reference = None
    if rank == 1:  # the reference arm returns at once on ranks > 0
        bench.run_reference(Args())
        ran_reference = False
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, e2e, value, ran_reference))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, e2e, value, _ in res:
        assert ms == 15.0 and e2e == 20.0  # the slowest rank's times on every rank
        assert value == pytest.approx(1000 * 4 * 2 / 0.015)
