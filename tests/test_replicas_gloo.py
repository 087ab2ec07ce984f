"""Multi-GPU runs of bench.py are independent replicas (one design per GPU, no collective on the data
path); the only cross-rank step is the timing reduction.  Two gloo ranks on the CPU check it: the job
time is the slowest rank's, the throughput counts every rank's iterations, and the reference arm does
its work on rank 0 only."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    times = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * (rank + 1)], world, "cpu")
    out[rank] = (times, bench.job_throughput(world, 5, times[0]))
    dist.barrier()
    if rank == 1:   # the reference arm returns at once on other ranks
        class A:
            config, steps, warmup, gpus = "c0", 1, 1, world
        out["ref_rank1"] = bench.run_reference_arm(A())
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    world, port = 2, 29611
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        times, thr = res[r]
        assert times == [2.0, 10.0, 1.0]
        assert thr == pytest.approx(2 * 5 / 2.0)
    assert res["ref_rank1"] == 0
