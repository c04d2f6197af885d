"""The N > 1 bench path on CPU: two gloo ranks on 127.0.0.1.  Each GPU runs an independent replica
of the workload (rays, pixels and requests need no exchange), so the only collective is the
max-over-ranks of the step times; the reference arm runs on rank 0 alone."""
import os
import socket
import sys
import types

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # per-rank step times: the slowest rank's time is the job's time
        got = bench.max_over_ranks([10.0 + rank, 20.0 - 3 * rank], dist, "cpu")
        # the reference arm: ranks other than 0 return at once without work
        ran = bench.run_reference(types.SimpleNamespace(ref_sample=1, warmup=0, steps=0), rank, world) if rank else None
        out[rank] = (got, ran)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_max_over_ranks_and_reference_arm():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(worker, args=(world, free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        got, ran = res[rank]
        assert got == [11.0, 20.0]
        assert ran is None


def test_single_rank_max_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5], None, "cpu") == [1.5, 2.5]
