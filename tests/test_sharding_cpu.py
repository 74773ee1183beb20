"""The multi-GPU far-field path on CPU: world_size 2 over gloo.

bench.py shards the focal plane by row blocks (each rank its own n-row tile of
a taller window, pillars replicated, no data-path collective) and reduces the
per-rank timings with a max over ranks. This runs that logic in two gloo
processes: the tiles computed per rank (with the oracle standing in for the
kernel, which the GPU tests check separately) must equal the corresponding
rows of the whole window, and the timing reduction must return the max.
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from celeris_b200.workloads import small_aperture


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, n, W, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from oracle import farfield as F

        a = small_aperture(97, seed=5)
        cy = bench.shard_center(rank, n, W)
        tile = F.rs_field(a.px, a.py, a.t, 0.0, cy, a.focal_um, a.k, n, W)
        m = bench.max_over_ranks(world, 10.0 + rank)
        tiles = [None] * world
        dist.all_gather_object(tiles, (rank, cy, tile, m))
        if rank == 0:
            out.put(tiles)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_row_block_shards_tile_the_window_and_max_reduces():
    world, n, W = 2, 6, 1.5
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(world, _free_port(), n, W, q), nprocs=world, join=True,
                       start_method="spawn")
    tiles = q.get()
    assert [t[3] for t in tiles] == [10.0 + world - 1] * world
    # the whole 2n-row window, evaluated densely
    a = small_aperture(97, seed=5)
    step = 2 * W / (n - 1)
    rows = -W + np.arange(world * n) * step
    cols = -W + np.arange(n) * step
    fy, fx = np.meshgrid(rows, cols, indexing="ij")
    R = np.sqrt((fx[..., None] - a.px) ** 2 + (fy[..., None] - a.py) ** 2 + a.focal_um ** 2)
    E = (a.t * np.exp(1j * a.k * R) / R).sum(-1)
    for rank, cy, tile, _ in tiles:
        ref = E[rank * n:(rank + 1) * n]
        assert np.max(np.abs(tile - ref)) <= 1e-11 * np.max(np.abs(E))
