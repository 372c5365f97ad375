"""render_distributed on the one GPU a call gets: a process group of one rank
over NCCL gives the single-GPU render bit for bit (the reduce and the count
weights are exact).  More ranks need more GPUs; the exchange step itself is
covered on CPU by tests/test_multirank.py."""
import datetime
import socket

import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes
from pathtracingtutorial_b200.distributed import render_distributed

pytestmark = pytest.mark.gpu


def test_one_rank_equals_single_gpu_render():
    import torch.distributed as dist
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sa = scenes.cornell_box(width=64, height=48)
        sc = sa.scene()
        sc.build_accel()
        sc.upload_to_device(0)
        img = render_distributed(sc, 32)
        assert sc.info()["frame_count"] == 32 // sa.sample_per_frame   # as a single-GPU render leaves it
        ref = pt.render(sc, 32)
        assert img.shape == ref.shape and img[..., :3].mean() > 0
        assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    finally:
        dist.destroy_process_group()
