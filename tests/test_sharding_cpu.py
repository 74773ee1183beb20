"""The multi-GPU split of one far field, one adjoint and one RCWA batch
(celeris_b200.multigpu) on CPU: world_size 2 over gloo.

The partition, padding, gather, all-reduce and reassembly are the product's
own code; only the per-block evaluation, which needs a GPU, is the oracle here
(the GPU tests run the same blocks through the kernels). Each result must equal
the one-rank evaluation of the whole grid / batch. bench.py's max-over-ranks
timing reduction is checked too.
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from celeris_b200 import multigpu as MG
from celeris_b200.workloads import small_aperture

N, W = 7, 1.5  # 7 rows over 2 ranks: blocks of 4 and 3 rows (the padded gather)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _Grid:
    def __init__(self, a):
        self.n, self.W, self.z, self.k, self.cx, self.cy = N, W, a.focal_um, a.k, 0.2, -0.1


def _cells():
    return [dict(period_um=0.4, wavelength_um=0.55 + 0.01 * i, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0,
                 fill_x=0.3 + 0.05 * i, thickness_um=0.5, Mx=1 + (i % 2)) for i in range(5)]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from oracle import farfield as F
        from oracle import rcwa as RO

        a = small_aperture(97, seed=5)
        g = _Grid(a)
        full = F.rs_field(a.px, a.py, a.t, g.cx, g.cy, g.z, g.k, N, W)

        def field_rows(r0, nr):  # the oracle stands in for celeris_rs_field_rows_dev
            return torch.from_numpy(F.rs_field(a.px, a.py, a.t, g.cx, g.cy, g.z, g.k, N, W, rows=(r0, r0 + nr))
                                    [r0:r0 + nr].copy())

        E = MG.rs_field_distributed(a.px, a.py, a.t, g, group=None, compute=field_rows).numpy()

        v = np.random.default_rng(3).standard_normal((N, N)) + 1j * np.random.default_rng(4).standard_normal((N, N))

        def adj_rows(r0, nr, vr):  # the adjoint over rows [r0, r0 + nr) only
            vm = np.zeros((N, N), complex)
            vm[r0:r0 + nr] = vr.numpy()
            return torch.from_numpy(F.rs_adjoint(a.px, a.py, g.cx, g.cy, g.z, g.k, N, W, vm))

        G = MG.rs_adjoint_distributed(a.px, a.py, torch.from_numpy(v), g, compute=adj_rows).numpy()

        def solve(cells):  # the oracle stands in for celeris_rcwa_batch
            res = []
            for c in cells:
                res += [RO.solve_cell(**c, Ex0=1.0, Ey0=0.0), RO.solve_cell(**c, Ex0=0.0, Ey0=1.0)]
            return res, np.zeros(len(cells), dtype=np.int32)

        res, info = MG.rcwa_batch_distributed(_cells(), solve=solve)
        m = bench.max_over_ranks(world, 10.0 + rank)
        got = [None] * world
        dist.all_gather_object(got, (rank, E, G, [r["tx0"] for r in res], list(info), m))
        if rank == 0:
            out.put((got, full, F.rs_adjoint(a.px, a.py, g.cx, g.cy, g.z, g.k, N, W, v)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_distributed_field_adjoint_and_rcwa_match_one_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(world, _free_port(), q), nprocs=world, join=True, start_method="spawn")
    got, full, adj = q.get()
    from oracle import rcwa as RO

    want_t = []
    for c in _cells():
        want_t += [RO.solve_cell(**c, Ex0=1.0, Ey0=0.0)["tx0"], RO.solve_cell(**c, Ex0=0.0, Ey0=1.0)["tx0"]]
    for rank, E, G, tx, info, m in got:
        # every rank holds the whole field, the whole adjoint and every cell's results
        assert E.shape == (N, N)
        assert np.array_equal(E, full), rank
        assert np.max(np.abs(G - adj)) <= 1e-12 * np.max(np.abs(adj)), rank
        assert tx == want_t and info == [0] * 5
        assert m == 10.0 + world - 1


def test_row_blocks_cover_the_grid():
    for n in (1, 2, 7, 161, 1024):
        for parts in (1, 2, 3, 8):
            b = MG.split_rows(n, parts)
            assert len(b) == parts
            assert b[0][0] == 0 and sum(nr for _, nr in b) == n
            assert all(b[i][0] + b[i][1] == b[i + 1][0] for i in range(parts - 1))
            assert max(nr for _, nr in b) - min(nr for _, nr in b) <= 1


def test_rcwa_cells_shard_by_flop_weight():
    """The RCWA batch splits over ranks by n^3 weight: every cell exactly once,
    loads within one largest cell of each other."""
    from celeris_b200.workloads import rcwa_uneven_4096

    cells = rcwa_uneven_4096()
    for world in (1, 2, 3, 8):
        parts = MG.shard_cells(cells, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cells)))
        w = [MG.cell_weight(c) for c in cells]
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(w)
