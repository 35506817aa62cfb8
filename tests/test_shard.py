"""The multi-GPU frame split on the host: the ranks' tiles partition the frame; two gloo ranks
render their tiles of a small frame with the CPU oracle and reduce their images to rank 0, and the
result equals one process rendering the whole frame bit for bit; and a rank that does not join the
reduction (it leaves, or it stalls) ends the waiting rank's reduction with an error within the
process group's timeout. CPU only (world size 2)."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from kernel_fixtures import lamp_scene
from lumenwright_b200 import layout as L
from lumenwright_b200 import shard

W, H = 20, 11  # not a multiple of the 8x4 tile


def frame_scene():
    ks = lamp_scene(L.EMITTER_SAMPLING_ONE, True)
    p = ks.params
    p["frame"] = [W, H, 0, 3]
    p["cam_pos"] = [8.0, 12.0, 8.0, 0.9]
    p["cam_fwd"] = [0.0, -1.0, 0.0, 1.5]
    p["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    p["sun_dir"] = [0.3, 0.9, 0.316, 0.9995]
    p["sun_color"] = [1.0, 0.9, 0.8, 0.03]
    return ks


def frame_mean(spp):
    from oracle import oracle as O
    ks = frame_scene()
    return O.OracleScene(*ks.buffers()).render_mean(0, 0, W, H, spp)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
@pytest.mark.parametrize("size", [(1, 1), (7, 3), (8, 4), (20, 11), (1280, 720)])
def test_the_ranks_tiles_partition_the_frame(world, size):
    w, h = size
    masks = np.stack([shard.tile_mask(w, h, r, world) for r in range(world)])
    assert np.array_equal(masks.sum(0), np.ones((h, w)))
    assert shard.frame_spp(1024, world) == 1024 * world


def worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local = np.where(shard.tile_mask(W, H, rank, world)[..., None], frame_mean(8), np.float32(0.0))
    m = shard.reduce_images(local.astype(np.float32), dist)
    if rank == 0:
        np.save(out, m)
    dist.barrier()
    dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_ranks_give_the_single_process_frame(tmp_path):
    out = str(tmp_path / "m.npy")
    mp.start_processes(worker, args=(2, free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    want = frame_mean(8)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def leaving_worker(rank, world, port, out, mode):
    import datetime
    import time

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        # This rank never joins the reduction: it leaves between steps with nothing in flight, or
        # it stalls past the process group's timeout before leaving.
        if mode == "stalls":
            time.sleep(12.0)
        dist.destroy_process_group()
        return
    t0 = time.monotonic()
    try:
        shard.reduce_images(np.ones((2, 3, 3), np.float32), dist)
        result = "none"
    except Exception as e:  # the reduction's error
        result = type(e).__name__
    with open(out, "w") as f:
        f.write(f"{result} {time.monotonic() - t0:.1f}")


@pytest.mark.parametrize("mode", ["leaves", "stalls"])
def test_a_rank_that_does_not_join_ends_the_reduction_with_an_error(tmp_path, mode):
    # Failure detection on the host: the rank left waiting in the reduction gets an error (at once
    # when its peer has left, after the process group's 5 s timeout when its peer stalls) instead
    # of waiting for good.
    out = str(tmp_path / "r.txt")
    mp.start_processes(leaving_worker, args=(2, free_port(), out, mode), nprocs=2, join=True, start_method="spawn")
    result, seconds = open(out).read().split()
    assert result != "none"
    assert float(seconds) < 11.0
