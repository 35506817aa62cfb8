"""Multi-GPU rendering of one hq frame: one process and context per GPU, each rendering every sample
of its share of the frame's 8x4-pixel tiles (rank r of N takes tiles r, r + N, r + 2N, ... row by
row, which spreads the sky and the terrain over the ranks), then one SUM reduce of the
accumulators to rank 0.

Every (pixel, sample) is independent (the random stream is keyed by pixel, sample index and seed,
crates/lumenwright-kernel/src/rng.rs:23-27) and a pixel's Kahan sums depend on its own samples
only, so each pixel's record on its rank is the one a single GPU rendering the whole frame makes,
bit for bit; every other rank holds zeros there, and adding zeros is exact. The reduced frame is
therefore the single-GPU frame bit for bit. Under weak scaling the frame's spp grows with the
ranks (each rank renders 1/N of the pixels at N times the spp). The reduction runs over whatever
process group is given: NCCL over NVLink on GPUs (on the device accumulators, on the library's
stream), gloo on the host in the tests.
"""

import numpy as np


def tile_mask(width: int, height: int, rank: int, world: int) -> np.ndarray:
    """(height, width) booleans: the pixels of rank `rank`'s tiles (the library's
    lw_render_device_shard with shard = rank, shards = world)."""
    tiles_x = (width + 7) // 8
    y, x = np.mgrid[0:height, 0:width]
    tile = (y // 4) * tiles_x + x // 8
    return tile % world == rank


def frame_spp(spp: int, world: int) -> int:
    """The frame's samples per pixel under weak scaling: each rank's work is a whole frame's at
    `spp`."""
    return spp * world


class _DeviceRecords:
    """A device buffer seen through the CUDA array interface (zero-copy into torch)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3,
                                         "strides": None}


def accumulator_tensor(ctx):
    """The context's device accumulator records (w * h * 8 floats) as a torch tensor sharing its
    memory."""
    import torch
    ptr, w, h = ctx.accumulator_device()
    return torch.as_tensor(_DeviceRecords(ptr, w * h * 8), device=f"cuda:{ctx.device}")


def reduce_accumulator(ctx, dist):
    """SUM-reduces every rank's accumulator records onto rank 0's, in place, ordered after the
    renders queued on the context's stream (the collective runs with that stream current, so
    anything queued on it afterwards, a timing mark included, follows the collective)."""
    import torch
    t = accumulator_tensor(ctx)
    with torch.cuda.stream(torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{ctx.device}")):
        dist.reduce(t, 0, op=dist.ReduceOp.SUM)


def render_hq_sharded(ctx, frame, dist, rank: int, world: int, spp=None):
    """The frame through the public calls with host buffers, split over the ranks: the scene and
    sky copied in, this rank's tiles rendered, the accumulators reduced to rank 0, which reads the
    image back ((h, w, 3) float32); the other ranks get None."""
    p = frame.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    ctx.upload_hq_scene(frame.scene)
    ctx.upload_sky(frame.sky)
    ctx.clear_accumulator(w, h)
    ctx.render_device_shard(p, 0, int(spp or frame.spp), rank, world)
    reduce_accumulator(ctx, dist)
    return ctx.read_accumulator(w, h) if rank == 0 else None


def reduce_images(local: np.ndarray, dist, device=None) -> np.ndarray:
    """The frame on rank 0 from every rank's image of its own tiles (zeros elsewhere): one SUM
    reduce of (h, w, 3) float32 images. Other ranks get None."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(local, np.float32))
    if device is not None:
        t = t.to(device)
    dist.reduce(t, 0, op=dist.ReduceOp.SUM)
    if dist.get_rank() != 0:
        return None
    return t.cpu().numpy()
