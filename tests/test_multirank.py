"""The multi-GPU path's host logic on CPU ranks (gloo, world size 2): each rank takes its own
ray range (bench.rank_rays) -- together exactly the first 2R rays of the single-process
stream, with no overlap -- and the job time is the slowest rank's (bench.max_over_ranks)."""

import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, count, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rays = torch.from_numpy(bench.rank_rays(rank, count))
        gathered = [torch.empty_like(rays) for _ in range(world)]
        dist.all_gather(gathered, rays)
        slowest = bench.max_over_ranks(0.5 + rank, dist, "cpu")
        if rank == 0:
            out.put((torch.cat(gathered).numpy(), slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_rays_and_take_the_slowest_time():
    import bench

    world, count = 2, 1000
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, count, out)) for r in range(world)]
    for p in procs:
        p.start()
    rays, slowest = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(rays, bench.rank_rays(0, world * count))
    assert slowest == 1.5
    assert bench.max_over_ranks(0.25, None, "cpu") == 0.25
