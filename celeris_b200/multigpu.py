"""One far-field grid, one adjoint or one RCWA batch split over several GPUs.

The reference has no multi-GPU code; its only split is of focal rows over host
threads (parallel_rows, src/celeris/analysis/focal.cpp:19-29). Here the same
independence carries over to devices:

  far field   rows of the focal grid are independent: each device computes a
              contiguous block of rows (celeris_rs_field_rows_dev) with every
              pillar replicated, and the blocks are gathered in row order;
  adjoint     each device sums over its own rows only
              (celeris_rs_adjoint_rows_dev); the per-pillar complex sums are
              added up (one all-reduce);
  RCWA batch  cells are independent: they are split by flop weight n^3
              (greedy longest-first), each device solves its share in one
              batched call, and the (small) results are gathered.

Two launch models:
  * one process, several devices - ``rs_field_multi``, ``rs_adjoint_multi``,
    ``rcwa_batch_multi``: one host thread per device; the blocks meet on the
    first device (torch peer copies, no library kernel reads a peer's memory);
  * one process per GPU under torch.distributed - ``rs_field_distributed``,
    ``rs_adjoint_distributed``, ``rcwa_batch_distributed``: all_gather of the
    row blocks, all_reduce of the adjoint sums, all_gather_object of the RCWA
    results (NCCL on GPUs; the gloo backend runs the same code on CPU).

No kernel here waits on another device, and nothing uses TMA multicast.
"""
from __future__ import annotations

import threading

import numpy as np

from . import capi


# ---- partitions -------------------------------------------------------------------
def split_rows(n: int, parts: int) -> list[tuple[int, int]]:
    """Contiguous row blocks (row0, nrows) of an n-row grid over `parts` workers,
    sizes differing by at most one (the first n % parts blocks one row longer)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    base, extra = divmod(int(n), parts)
    out, r0 = [], 0
    for p in range(parts):
        nr = base + (1 if p < extra else 0)
        out.append((r0, nr))
        r0 += nr
    return out


def cell_weight(cell) -> int:
    """Flop weight of one cell solve: n^3, n = 2 (2Mx + 1)(2My + 1)."""
    if isinstance(cell, dict):
        mx, my = cell["Mx"], cell.get("My", cell["Mx"])
    else:
        mx, my = cell.Mx, cell.My
    return (2 * (2 * mx + 1) * (2 * my + 1)) ** 3


def shard_cells(cells, world: int) -> list[list[int]]:
    """Indices of the cells each of `world` workers solves: greedy
    longest-first by n^3 onto the least-loaded worker; every cell lands on
    exactly one worker, each list in ascending order."""
    w = [cell_weight(c) for c in cells]
    parts, loads = [[] for _ in range(world)], [0] * world
    for i in sorted(range(len(cells)), key=lambda i: (-w[i], i)):
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += w[i]
    return [sorted(p) for p in parts]


# ---- device kernels of one row block ------------------------------------------------
def _ptr(t):
    import ctypes

    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import ctypes

    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def rows_field_dev(px, py, t, grid, form, row0, nrows):
    """Rows [row0, row0 + nrows) of the far field of `grid` on the tensors' device."""
    import torch

    E = torch.empty((nrows, grid.n), dtype=torch.complex128, device=t.device)
    capi.check(capi.load().celeris_rs_field_rows_dev(form, _ptr(px), _ptr(py), _ptr(t), int(px.numel()), grid.cx,
                                                     grid.cy, grid.z, grid.k, grid.n, grid.W, int(row0), int(nrows),
                                                     _ptr(E), None, _stream()))
    return E


def rows_adjoint_dev(px, py, v_rows, grid, form, row0, nrows):
    """The adjoint sum over rows [row0, row0 + nrows) only; v_rows: (nrows, n)."""
    import torch

    out = torch.empty(px.numel(), dtype=torch.complex128, device=v_rows.device)
    v_rows = v_rows.contiguous()
    capi.check(capi.load().celeris_rs_adjoint_rows_dev(form, _ptr(px), _ptr(py), int(px.numel()), grid.cx, grid.cy,
                                                       grid.z, grid.k, grid.n, grid.W, int(row0), int(nrows),
                                                       _ptr(v_rows), _ptr(out), _stream()))
    return out


# ---- one process, several devices --------------------------------------------------
def _run_threads(fns):
    """Run fns[i]() on thread i; re-raise the first failure."""
    res, errs = [None] * len(fns), [None] * len(fns)

    def work(i):
        try:
            res[i] = fns[i]()
        except BaseException as e:  # noqa: BLE001 - re-raised below
            errs[i] = e

    th = [threading.Thread(target=work, args=(i,)) for i in range(len(fns))]
    for x in th:
        x.start()
    for x in th:
        x.join()
    for e in errs:
        if e is not None:
            raise e
    return res


def rs_field_multi(px, py, t, grid, form=capi.FORM_PLAIN_F64, devices=None):
    """The far field of `grid` with its rows split over `devices` (CUDA device
    indices; default all visible). Inputs: float64 px, py and complex128 t
    (numpy or torch). Returns the (n, n) complex128 field on devices[0]."""
    import torch

    devices = list(range(torch.cuda.device_count())) if devices is None else list(devices)
    blocks = split_rows(grid.n, len(devices))
    for d in set(devices):  # inputs produced on the callers' streams are complete
        torch.cuda.synchronize(d)

    def one(d, r0, nr):
        def f():
            # a stream of this thread's own: the library keeps one workspace
            # arena per (device, stream), so two threads must not share one
            with torch.cuda.device(d), torch.cuda.stream(torch.cuda.Stream(device=d)):
                dev = torch.device("cuda", d)
                a = [torch.as_tensor(v).to(dev) for v in (px, py, t)]
                E = rows_field_dev(a[0], a[1], a[2], grid, form, r0, nr) if nr > 0 else None
                torch.cuda.current_stream().synchronize()
                return E
        return f

    parts = _run_threads([one(d, r0, nr) for d, (r0, nr) in zip(devices, blocks)])
    home = torch.device("cuda", devices[0])
    return torch.cat([p.to(home) for p in parts if p is not None], dim=0)


def rs_adjoint_multi(px, py, v, grid, form=capi.FORM_PLAIN_F64, devices=None):
    """The adjoint sum_p conj(g_pj) v_p with the pixel rows split over `devices`:
    each device sums its rows; the per-pillar sums are added on devices[0]."""
    import torch

    devices = list(range(torch.cuda.device_count())) if devices is None else list(devices)
    blocks = split_rows(grid.n, len(devices))
    v = torch.as_tensor(v)
    for d in set(devices):
        torch.cuda.synchronize(d)

    def one(d, r0, nr):
        def f():
            with torch.cuda.device(d), torch.cuda.stream(torch.cuda.Stream(device=d)):
                dev = torch.device("cuda", d)
                a = [torch.as_tensor(x).to(dev) for x in (px, py)]
                out = rows_adjoint_dev(a[0], a[1], v[r0:r0 + nr].to(dev), grid, form, r0, nr) if nr > 0 else None
                torch.cuda.current_stream().synchronize()
                return out
        return f

    parts = _run_threads([one(d, r0, nr) for d, (r0, nr) in zip(devices, blocks)])
    home = torch.device("cuda", devices[0])
    total = None
    for p in parts:
        if p is not None:
            total = p.to(home) if total is None else total + p.to(home)
    return total


def rcwa_batch_multi(cells, devices=None):
    """capi.rcwa_batch with the cells split over `devices` by n^3 weight.
    Returns (results, info) in the order of `cells` (2 results per cell: X, Y)."""
    import torch

    devices = list(range(torch.cuda.device_count())) if devices is None else list(devices)
    parts = shard_cells(cells, len(devices))

    def one(d, idx):
        def f():
            if not idx:
                return [], np.zeros(0, dtype=np.int32)
            torch.cuda.set_device(d)
            return capi.rcwa_batch([cells[i] for i in idx])
        return f

    outs = _run_threads([one(d, idx) for d, idx in zip(devices, parts)])
    res = [None] * (2 * len(cells))
    info = np.zeros(len(cells), dtype=np.int32)
    for idx, (r, inf) in zip(parts, outs):
        for k, i in enumerate(idx):
            res[2 * i], res[2 * i + 1] = r[2 * k], r[2 * k + 1]
            info[i] = inf[k]
    return res, info


# ---- one process per GPU (torch.distributed) ----------------------------------------
def _world(group):
    import torch.distributed as dist

    return dist.get_world_size(group), dist.get_rank(group)


def rs_field_distributed(px, py, t, grid, form=capi.FORM_PLAIN_F64, group=None, compute=None):
    """The far field of `grid` computed by all ranks of `group` together: rank r
    computes rows split_rows(n, world)[r] and an all_gather returns the whole
    (n, n) complex128 field on every rank. `compute(row0, nrows)` evaluates one
    block (default: the GPU kernel on this rank's current device, inputs copied
    there); the backend's device is the tensors' device."""
    import torch
    import torch.distributed as dist

    world, rank = _world(group)
    blocks = split_rows(grid.n, world)
    r0, nr = blocks[rank]
    if compute is None:
        dev = torch.device("cuda", torch.cuda.current_device())
        a = [torch.as_tensor(v).to(dev) for v in (px, py, t)]

        def compute(row0, nrows):
            return rows_field_dev(a[0], a[1], a[2], grid, form, row0, nrows)

    mine = compute(r0, nr) if nr > 0 else None
    rows_max = max(b[1] for b in blocks)
    dev = mine.device if mine is not None else (torch.device("cuda", torch.cuda.current_device())
                                                if dist.get_backend(group) == "nccl" else torch.device("cpu"))
    # equal-sized blocks for all_gather: real and imaginary parts as float64
    buf = torch.zeros((rows_max, grid.n, 2), dtype=torch.float64, device=dev)
    if mine is not None:
        buf[:nr] = torch.view_as_real(mine.to(dev))
    got = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(got, buf, group=group)
    full = torch.cat([got[p][:blocks[p][1]] for p in range(world)], dim=0)
    return torch.view_as_complex(full.contiguous())


def rs_adjoint_distributed(px, py, v, grid, form=capi.FORM_PLAIN_F64, group=None, compute=None):
    """The adjoint over the whole grid by all ranks of `group`: rank r sums over
    its rows (v may be the whole (n, n) pixel array or only this rank's rows),
    and one all_reduce adds the per-pillar complex sums (returned on every
    rank). `compute(row0, nrows, v_rows)` evaluates one block (default: the GPU
    kernel)."""
    import torch
    import torch.distributed as dist

    world, rank = _world(group)
    r0, nr = split_rows(grid.n, world)[rank]
    v = torch.as_tensor(v)
    v_rows = v[r0:r0 + nr] if v.shape[0] == grid.n else v
    if compute is None:
        dev = torch.device("cuda", torch.cuda.current_device())
        a = [torch.as_tensor(x).to(dev) for x in (px, py)]

        def compute(row0, nrows, vr):
            return rows_adjoint_dev(a[0], a[1], vr.to(dev), grid, form, row0, nrows)

    npil = int(np.asarray(px).shape[0]) if not hasattr(px, "numel") else int(px.numel())
    part = compute(r0, nr, v_rows) if nr > 0 else None
    dev = part.device if part is not None else (torch.device("cuda", torch.cuda.current_device())
                                                if dist.get_backend(group) == "nccl" else torch.device("cpu"))
    acc = torch.zeros((npil, 2), dtype=torch.float64, device=dev)
    if part is not None:
        acc += torch.view_as_real(part.to(dev))
    dist.all_reduce(acc, op=dist.ReduceOp.SUM, group=group)
    return torch.view_as_complex(acc.contiguous())


def rcwa_batch_distributed(cells, group=None, solve=None):
    """capi.rcwa_batch over all ranks of `group`: rank r solves the cells
    shard_cells(cells, world)[r] in one batched call (`solve(cells)` -> (results,
    info), default capi.rcwa_batch), and all_gather_object returns every
    cell's (X, Y) results and info, in the order of `cells`, on every rank."""
    import torch.distributed as dist

    world, rank = _world(group)
    parts = shard_cells(cells, world)
    solve = capi.rcwa_batch if solve is None else solve
    mine = parts[rank]
    r, inf = solve([cells[i] for i in mine]) if mine else ([], np.zeros(0, dtype=np.int32))
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, list(r), [int(x) for x in inf]), group=group)
    res = [None] * (2 * len(cells))
    info = np.zeros(len(cells), dtype=np.int32)
    for idx, rr, ii in gathered:
        for k, i in enumerate(idx):
            res[2 * i], res[2 * i + 1] = rr[2 * k], rr[2 * k + 1]
            info[i] = ii[k]
    return res, info
