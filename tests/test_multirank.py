"""The N > 1 path of bench.py on CPU: two gloo ranks, timings reduced with a
max over ranks (the slowest replica sets the step time), whole-job value."""
import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms, e2e = bench.max_over_ranks([1.0 + rank, 10.0 - rank], world)
        out[rank] = (ms, e2e, bench.aggregate_value(1e9, ms, world))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_aggregate():
    world = 2
    port = 29500 + (os.getpid() % 1000)
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        ms, e2e, value = out[r]
        assert ms == 2.0 and e2e == 10.0  # max over ranks, element-wise
        assert value == pytest.approx(world * 1e9 / 2e-3 / 1e9)
