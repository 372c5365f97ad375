"""Multi-rank plumbing on CPU (gloo, world size 2): bench.py's disjoint sample
ranges per rank and max-time / sum-rays reduction, and the frame split and
image reduction of pathtracingtutorial_b200.distributed.render_distributed."""
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


def test_frame_ranges_partition_the_frames():
    from pathtracingtutorial_b200.distributed import frame_range
    for frames in (0, 1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            got = [frame_range(r, world, frames) for r in range(world)]
            assert sum(c for _, c in got) == frames
            assert all(got[i][0] + got[i][1] == got[i + 1][0] for i in range(world - 1))
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        frame_range(2, 2, 10)


def _reduce_worker(rank, world, port, out):
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    from pathtracingtutorial_b200.distributed import frame_range, reduce_to_root
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    frames, spf = 11, 4
    first, count = frame_range(rank, world, frames)
    mean = torch.from_numpy(np.random.default_rng(rank).uniform(0, 1, (3, 5, 4)).astype(np.float32))
    weighted = mean * float(count * spf)
    reduce_to_root(weighted, dist)
    out[rank] = (first, count, (weighted / float(frames * spf)).numpy() if rank == 0 else None)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_image_reduction():
    """The exchange step of render_distributed on CPU tensors (gloo): rank 0
    ends with the sample-count-weighted mean of the ranks' images."""
    import numpy as np
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_reduce_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    (f0, c0, img), (f1, c1, _) = out[0], out[1]
    assert (f0, c0, f1, c1) == (0, 6, 6, 5)
    means = [np.random.default_rng(r).uniform(0, 1, (3, 5, 4)).astype(np.float32) for r in range(2)]
    expect = (means[0] * 24.0 + means[1] * 20.0) / 44.0
    assert np.allclose(img, expect, rtol=1e-6, atol=1e-7)
