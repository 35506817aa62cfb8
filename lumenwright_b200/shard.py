"""Multi-GPU sharding of one hq frame: one process per GPU, each rendering its own range of sample
indices of the whole frame, then one reduction of the per-pixel means to rank 0.

Every (pixel, sample) is independent (the random stream is keyed by pixel, sample index and seed,
crates/lumenwright-kernel/src/rng.rs:23-27), so contiguous sample ranges per rank give exactly the
samples a single GPU would draw, and the frame is the mean of the ranks' equally weighted means.
The reduction runs over whatever process group is given: NCCL over NVLink on GPUs, gloo on the
host in the tests.
"""

import numpy as np


def sample_range(rank: int, world: int, spp: int, step: int = 0):
    """(first sample index, count) of ``rank``'s share of step ``step``: each rank renders ``spp``
    samples of every pixel (weak scaling), the ranks' ranges side by side."""
    return (step * world + rank) * spp, spp


def reduce_means(local_mean: np.ndarray, dist, device=None) -> np.ndarray:
    """The frame's mean radiance on rank 0 from every rank's mean over an equal number of samples:
    one SUM reduce of (h, w, 3) float32 images, divided by the world size. Other ranks get None."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(local_mean, np.float32))
    if device is not None:
        t = t.to(device)
    dist.reduce(t, 0, op=dist.ReduceOp.SUM)
    if dist.get_rank() != 0:
        return None
    return (t / dist.get_world_size()).cpu().numpy()
