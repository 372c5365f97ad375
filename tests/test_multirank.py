"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): disjoint sample
ranges per rank and the max-time / sum-rays reduction."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    batches = 64
    f0 = bench.shard_first_frame(rank, batches)
    ms, rays = bench.combine_over_ranks(100.0 + 50.0 * rank, 1000 * (rank + 1), dist, "cpu")
    out[rank] = (f0, ms, rays)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_sharding_and_reduction():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    (f0a, msa, ra), (f0b, msb, rb) = out[0], out[1]
    # frames [0, 64) and [64, 128): the Sobol indices 4*f + i never overlap
    assert (f0a, f0b) == (0, 64)
    assert msa == msb == 150.0
    assert ra == rb == 3000.0
