"""One render split over the ranks of a torch.distributed process group.

The path shards by sample index: every rank holds the whole scene on its own
GPU and renders a disjoint, contiguous range of the render's frames (sample
passes), so the per-rank images are independent estimates over disjoint
sample indices.  The one exchange step is a reduce (SUM) to rank 0 of each
rank's mean image weighted by its sample count, over NCCL on CUDA tensors
(NVLink between the GPUs of a node); rank 0 divides by the total sample count.
With one rank the result is the single-GPU render bit for bit (the weights
and the division are exact powers of two for the usual samples per frame).
The reference renders on one GPU only (Part_2/src/renderer.cu:87-111).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._ffi import check, lib


def frame_range(rank: int, world: int, frames: int) -> tuple[int, int]:
    """(first frame, number of frames) of `rank`: `frames` split into `world`
    contiguous ranges whose sizes differ by at most one, lower ranks first."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(frames, world)
    return rank * base + min(rank, extra), base + (1 if rank < extra else 0)


def reduce_to_root(weighted, dist, group=None):
    """Sum the ranks' count-weighted images into rank 0's tensor (in place)."""
    dist.reduce(weighted, dst=dist.get_global_rank(group, 0) if group is not None else 0, op=dist.ReduceOp.SUM,
                group=group)
    return weighted


def render_distributed(scene, spp: int, group=None, renderer=None):
    """render(scene, spp) over the ranks of `group` (default: the world).
    Every rank calls it with the same scene and spp, its scene uploaded to its
    own device.  Returns the (H, W, 4) image on rank 0, None elsewhere.
    Afterwards every rank's scene stands at the frame count a single-GPU
    render of spp leaves (all of the render's frames), so a later render
    continues from the same sample index on every rank."""
    import torch
    import torch.distributed as dist
    from . import Renderer
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    spf = scene.settings().sample_per_frame
    frames = -(-int(spp) // spf)
    first, count = frame_range(rank, world, frames)
    r = renderer or Renderer(scene)
    r.reset_accumulation()
    scene.set_frame_count(first)
    cam = scene.camera
    h, w = int(cam["height"]), int(cam["width"])
    img = torch.zeros((h, w, 4), dtype=torch.float32, device=f"cuda:{r.film.device}")
    if count:
        r.render_frames(count)
        r.synchronize()   # the integrator's stream does not order with the copy's
        check(lib().pt_film_download_to(r.film._h, C.c_void_p(img.data_ptr()), 1))
        img *= float(count * spf)
    torch.cuda.synchronize(img.device)
    scene.set_frame_count(frames)
    reduce_to_root(img, dist, group)
    if rank != 0:
        return None
    img /= float(frames * spf)
    return img.cpu().numpy()
