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


def test_rcwa_cells_shard_by_flop_weight():
    """The RCWA batch splits over ranks by n^3 weight: every cell exactly once,
    loads within one largest cell of each other."""
    import bench
    from celeris_b200.workloads import rcwa_uneven_4096

    cells = rcwa_uneven_4096()
    for world in (1, 2, 3, 8):
        parts = bench.shard_cells(cells, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cells)))
        w = [(2 * (2 * c["Mx"] + 1) * (2 * c.get("My", c["Mx"]) + 1)) ** 3 for c in cells]
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(w)


def _rcwa_worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from celeris_b200.workloads import rcwa_uneven_4096

        parts = bench.shard_cells(rcwa_uneven_4096(), world)
        got = [None] * world
        dist.all_gather_object(got, (rank, parts[rank], bench.max_over_ranks(world, 1.0 + rank)))
        if rank == 0:
            out.put(got)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_rcwa_shards_agree_across_ranks():
    """Each gloo rank computes the same partition independently (no exchange
    needed to agree) and the timing reduction returns the slowest rank."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_rcwa_worker, args=(world, _free_port(), q), nprocs=world, join=True, start_method="spawn")
    got = q.get()
    parts = [g[1] for g in sorted(got)]
    assert sorted(parts[0] + parts[1]) == list(range(4096))
    assert not set(parts[0]) & set(parts[1])
    assert all(g[2] == float(world) for g in got)
