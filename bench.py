#!/usr/bin/env python
"""Benchmark of the CELERIS B200 hot path.

Headline (one JSON line on rank 0): RS terms/s of the far-field sum in the
chosen (FP32-compensated) form on the 785,456-pillar metalens with a 1024 x 1024
focal grid (+/-20 um at z = 1 mm, lambda 532 nm), with its error against the
FP64 form stated. A step is one evaluation of the whole focal grid. Secondary
objects on the same line: the plain FP64 form on the same workload, both forms
on the 70,688-pillar x 161^2 metalens, the roofline of the dominant kernel
against in-run measured pipe peaks, the reference's own CPU far-field timed on
this host (cpu_baseline), the end-to-end C-ABI call with host buffers (e2e),
RCWA cells/s when the RCWA kernels are present, and the SM clocks seen.

Multi-GPU (torchrun, one rank per GPU): the focal plane is sharded by row
blocks - each rank evaluates its own 1024 x 1024 tile of a taller focal window
(pillars replicated, no data-path collective): weak scaling. Timing is CUDA
events, barrier + synchronize around the timed region, max over ranks.

--impl reference times the reference's own CPU propagate_pillars (compiled from
its sources into oracle/_ref) on this host's cores, on bounded samples of the
same workload, and prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RS terms/s"
UNIT = "terms/s"
WORKLOAD = "metalens_785k_1024sq_f32c"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="celeris", choices=["celeris", "reference"])
    ap.add_argument("--quick", action="store_true", help="skip secondary measurements")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--case", default=None,
                    help="run one small named case and exit (ncu captures): ff785k_f32c_256, "
                         "ff785k_f64_128, ff70k_f32c, ff70k_f64, ff70k_adj, rcwa_library, rcwa_M<m>_<ncell>")
    ap.add_argument("--reps", type=int, default=2)
    return ap.parse_args()


# ---------------------------------------------------------------- distributed
def dist_init(n):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, x):
    """Max of a per-rank scalar over all ranks (NCCL on GPUs, gloo on CPU)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_center(rank, n, half_window_um):
    """Window centre y of rank `rank`'s n-row tile: the tiles of ranks 0..N-1
    are consecutive, disjoint row blocks of one taller focal window whose first
    row sits at -half_window (weak scaling, pillars replicated)."""
    step = 2.0 * half_window_um / (n - 1)
    return rank * n * step


def measure_rcwa_sharded(world, rank):
    """4096 uneven cells split over the ranks by flop weight (strong scaling):
    each rank solves its share in one batched call; max-over-ranks wall time of
    the warm call (the batch is synchronous, the host clock brackets the device
    work) gives the whole-job cells/s."""
    from celeris_b200 import capi
    from celeris_b200.multigpu import shard_cells
    from celeris_b200.workloads import rcwa_uneven_4096

    cells = rcwa_uneven_4096()
    mine = shard_cells(cells, world)[rank]
    cc = [capi.rcwa_cell(**cells[i]) for i in mine]
    capi.rcwa_batch(cc)  # tuning + graph capture
    barrier(world)
    t0 = time.perf_counter()
    res, info = capi.rcwa_batch(cc)
    dt = max_over_ranks(world, time.perf_counter() - t0)
    bad = max_over_ranks(world, float(np.sum(info != 0)))
    return {"value": len(cells) / dt, "unit": "cells/s", "s": dt, "ranks": world, "scaling": "strong",
            "sharding": "cells by n^3 weight, greedy longest-first", "failed_cells": int(bad)}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- workloads
def workload(rank):
    from celeris_b200.workloads import metalens_785k

    ap, g = metalens_785k()
    # rank r evaluates the r-th 1024-row tile of a taller focal window
    return ap, g, shard_center(rank, g.n, g.half_window_um)


def choose_cpu_sample(npil, seconds, rate_guess, threads):
    """Grid side n for a CPU sample of ~`seconds` (n >= threads so every host
    thread gets a row, as parallel_rows hands out rows)."""
    terms = seconds * rate_guess
    n = int(max(threads, min(1024, np.sqrt(terms / npil))))
    return max(n, 2)


def cpu_reference_sample(ap, g, seconds=12.0):
    """Time the reference's own CPU propagate_pillars on a bounded sample: all
    pillars, an n x n grid over the same window."""
    from oracle import farfield as F

    threads = F.ref_threads() or os.cpu_count()
    # calibrate on a tiny grid
    n0 = 2
    t0 = time.perf_counter()
    F.ref_propagate_pillars(ap.px, ap.py, ap.t, 0.0, 0.0, g.z_um, ap.wavelength_um, n0, g.half_window_um)
    dt0 = time.perf_counter() - t0
    rate0 = ap.npil * n0 * n0 / max(dt0, 1e-6) * max(1, threads // (n0))  # rough, rows cap threads
    n = choose_cpu_sample(ap.npil, seconds, rate0, threads)
    t0 = time.perf_counter()
    F.ref_propagate_pillars(ap.px, ap.py, ap.t, 0.0, 0.0, g.z_um, ap.wavelength_um, n, g.half_window_um)
    dt = time.perf_counter() - t0
    terms = ap.npil * n * n
    return {"value": terms / dt, "unit": UNIT, "cores": int(threads), "kind": "reference",
            "sample": f"{ap.npil} pillars x {n}x{n} pixels over the same +/-{g.half_window_um} um window "
                      f"({terms:.3e} terms, {dt:.2f} s), reference celeris::propagate_pillars FP64 CPU path "
                      f"compiled from its sources (-O3 -mavx2 -mfma), {threads} host threads"}


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    from oracle import farfield as F

    if F.ref_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_farfield.so not built"}))
        return
    ap, g, _ = workload(0)
    threads = F.ref_threads() or os.cpu_count()
    # size each step to ~5 s of host work
    n0 = max(2, threads)
    t0 = time.perf_counter()
    F.ref_propagate_pillars(ap.px, ap.py, ap.t, 0.0, 0.0, g.z_um, ap.wavelength_um, n0, g.half_window_um)
    rate = ap.npil * n0 * n0 / (time.perf_counter() - t0)
    n = choose_cpu_sample(ap.npil, 5.0, rate, threads)
    for _ in range(args.warmup):
        F.ref_propagate_pillars(ap.px, ap.py, ap.t, 0.0, 0.0, g.z_um, ap.wavelength_um, max(2, n // 4),
                                g.half_window_um)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        F.ref_propagate_pillars(ap.px, ap.py, ap.t, 0.0, 0.0, g.z_um, ap.wavelength_um, n, g.half_window_um)
        times.append(time.perf_counter() - t0)
    terms = ap.npil * n * n
    value = terms * len(times) / sum(times)
    sample = (f"each step: {ap.npil} pillars x {n}x{n} pixels ({terms:.3e} terms) of the "
              f"{g.n}x{g.n} workload, reference propagate_pillars FP64 CPU, {threads} host threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "pillars": ap.npil, "grid": f"{g.n}x{g.n}", "sampled_grid": f"{n}x{n}"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": int(threads), "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------- GPU arm
def measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool's B200s (MEASURED_PEAKS.json), else
    the pool's earlier measurement."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s, an earlier measurement on this pool)"


def profiles_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}.md")
    if not os.path.exists(path):
        return None
    for ln in open(path):
        if ln.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def timed_steps(fn, steps, stream, flush):
    import torch

    ms = []
    kms = []
    from celeris_b200 import capi

    for _ in range(steps):
        flush()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
        kms.append(capi.last_kernel_ms())
    return ms, kms


def rcwa_flops(cell, method="run"):
    """Algorithmic FP64 flops of one cell solve.
    method="reference": 240 n^3 (n = 2N, diagonal-aware count of the reference
    method: ep2 kp 4n^3, eigensolve 100n^3, interfaces 136n^3).
    method="run": the method this library runs. A mirror-symmetric cell at
    normal incidence (unrotated shape, theta = 0, Mx, My >= 1) solves the same
    steps in its two excited parity classes of order m = (Mx+1)(My+1) + Mx My:
    2 x 240 m^3, plus building M at full order (2 n^3) and projecting it, the
    layer kp and the half-space operators (4 x 16 x 8 m^2 per class). Other
    cells run the reference method.
    Both add n^3 for the Laurent inverse and the raster DFT on rasterised cells."""
    Mx, My = cell["Mx"], cell.get("My", cell["Mx"])
    N = (2 * Mx + 1) * (2 * My + 1)
    n = 2 * N
    sym = (cell.get("theta_rad", 0.0) == 0.0 and cell.get("rotation_rad", 0.0) == 0.0 and Mx >= 1 and My >= 1)
    if method == "run" and sym:
        m = (Mx + 1) * (My + 1) + Mx * My
        f = 2 * 240.0 * m ** 3 + 2.0 * n ** 3 + 2 * 4 * 16 * 8.0 * m * m
    else:
        f = 240.0 * n ** 3
    if cell.get("force_laurent") or cell.get("shape", 0) != 0:
        ng = cell.get("grid") or max(128, 8 * (2 * Mx + 1))
        M4 = 4 * Mx + 1
        f += n ** 3 + 8.0 * ng * ng * M4 + 8.0 * M4 * M4 * ng
    return f


def _oracle_cell_time(cell):
    import time as _t

    from oracle import rcwa as RO

    t0 = _t.perf_counter()
    RO.solve_cell(**cell, Ex0=1.0, Ey0=0.0)
    RO.solve_cell(**cell, Ex0=0.0, Ey0=1.0)  # the reference solves each polarization
    return _t.perf_counter() - t0


def rcwa_cpu_baseline(cells, budget_s=15.0):
    """The oracle port (numpy/LAPACK zgeev, one BLAS thread per worker) over all
    host cores, on a sample of the cells: per-M mean time -> whole-batch rate."""
    import concurrent.futures as cf
    import multiprocessing as mp

    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    os.environ.setdefault("MKL_NUM_THREADS", "1")
    workers = os.cpu_count() or 1
    byM = {}
    for c in cells:
        byM.setdefault(c["Mx"], []).append(c)
    per = max(1, min(workers, 8))
    sample = [c for M in sorted(byM) for c in byM[M][:per]]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with cf.ProcessPoolExecutor(max_workers=min(workers, len(sample)), mp_context=ctx) as ex:
        times = list(ex.map(_oracle_cell_time, sample))
    wall = time.perf_counter() - t0
    tM = {}
    for c, t in zip(sample, times):
        tM.setdefault(c["Mx"], []).append(t)
    total = sum(float(np.mean(tM[c["Mx"]])) for c in cells)
    rate = len(cells) / (total / workers)
    return {"value": rate, "unit": "cells/s", "cores": workers, "kind": "port",
            "sample": f"{len(sample)} cells ({per} per M) solved twice (X, Y) by the numpy/LAPACK restatement of "
                      f"solve_rcwa_2d, {workers} processes x 1 BLAS thread, {wall:.1f} s; per-M mean times "
                      f"scaled to the whole batch"}


def rcwa_library_cpu_baseline(cells):
    """The oracle port over the whole 64-cell library sweep, X and Y solved
    separately as the reference does (polarization.cpp:35-39), one cell per
    process over all host cores, one BLAS thread each."""
    import concurrent.futures as cf
    import multiprocessing as mp

    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    os.environ.setdefault("MKL_NUM_THREADS", "1")
    workers = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(max_workers=min(workers, len(cells)), mp_context=ctx) as ex:
        list(ex.map(_oracle_cell_time, cells[:min(workers, len(cells))]))  # start the workers, import numpy
        t0 = time.perf_counter()
        list(ex.map(_oracle_cell_time, cells))
        wall = time.perf_counter() - t0
    return {"value": len(cells) / wall, "unit": "cells/s", "cores": workers, "kind": "port",
            "sample": f"all {len(cells)} cells of the sweep, X and Y each solved by the numpy/LAPACK restatement of "
                      f"solve_rcwa_2d, {workers} processes x 1 BLAS thread, {wall:.2f} s wall"}


def measure_rcwa(peaks, quick=False, with_cpu=True, sampler=None):
    """RCWA cells/s. `sampler` (a ClockSampler) runs over both the 64-cell
    sweep and the uneven batch (polling nvidia-smi every 100 ms leaves the
    sweep's ~1 ms calls unchanged, measured on this B200)."""
    from celeris_b200 import capi
    from celeris_b200.workloads import rcwa_library_64, rcwa_uneven_4096

    out = {"metric": "RCWA cells/s (one cell = one geometry/wavelength solve, X and Y polarizations)",
           "unit": "cells/s", "dtype": "f64 complex"}
    # FP64 peak: the faster of the FMA pipe and the tensor cores (DMMA), both measured in-run
    p_fp64 = max(peaks["dfma_per_s"], peaks.get("dmma_fma_per_s", 0.0)) * 2.0
    if sampler is not None:
        sampler.start()
    lib = rcwa_library_64()
    lc = [capi.rcwa_cell(**c) for c in lib]
    capi.rcwa_batch(lc)
    t, tcpu = [], []
    for _ in range(11):  # host-synchronous calls: the median of 11 rides out host-side jitter
        t0, c0 = time.perf_counter(), time.process_time()
        capi.rcwa_batch(lc)
        t.append(time.perf_counter() - t0)
        tcpu.append(time.process_time() - c0)
    dt = float(np.median(t))
    t0 = time.perf_counter()
    for c in lc[:8]:
        capi.solve_rcwa_2d(c)
    per_cell = (time.perf_counter() - t0) / 8
    fl = sum(rcwa_flops(c) for c in lib)
    fl_ref = sum(rcwa_flops(c, "reference") for c in lib)
    out["library_64_M3"] = {"value": 64 / dt, "ms": 1e3 * dt, "per_cell_launch_cells_s": 1.0 / per_cell,
                            "batched_over_per_cell": per_cell / (dt / 64),
                            "roofline": {"bound": "fp64", "achieved": fl / dt, "peak": p_fp64, "unit": "FLOP/s",
                                         "frac": fl / dt / p_fp64,
                                         "flops": "of the method run (parity-class solve of mirror-symmetric cells)"},
                            "reference_method_flops_per_s": fl_ref / dt,
                            # per-call spread and host CPU time (process, all threads): a wall time far
                            # above the CPU time is time the calling thread spent waiting, not working
                            "calls_ms": {"min": 1e3 * min(t), "median": 1e3 * dt, "max": 1e3 * max(t),
                                         "cpu_median": 1e3 * float(np.median(tcpu))}}
    if with_cpu:
        try:
            out["library_64_M3"]["cpu_baseline"] = rcwa_library_cpu_baseline(lib)
        except Exception as exc:
            out["library_64_M3"]["cpu_baseline"] = {"unavailable": str(exc)[:200]}
    if not quick:
        cells = rcwa_uneven_4096()
        cc = [capi.rcwa_cell(**c) for c in cells]
        # first call: tunes the CTA sizes of new bucket shapes and captures the
        # batch graph; later calls with the same shapes replay it
        t0 = time.perf_counter()
        res, info = capi.rcwa_batch(cc)
        first = time.perf_counter() - t0
        warm = []
        for _ in range(2):
            t0 = time.perf_counter()
            res, info = capi.rcwa_batch(cc)
            warm.append(time.perf_counter() - t0)
        dt2 = min(warm)
        fl2 = sum(rcwa_flops(c) for c in cells)
        fl2_ref = sum(rcwa_flops(c, "reference") for c in cells)
        out["uneven_4096_M3to7_grid256"] = {
            "value": len(cells) / dt2, "s": dt2, "first_call_s": first,
            "first_call_cells_s": len(cells) / first, "failed_cells": int(np.sum(info != 0)),
            "max_abs_R_plus_T_minus_1": float(max(abs(r["R"] + r["T"] - 1.0) for r in res)),
            "roofline": {"bound": "fp64", "achieved": fl2 / dt2, "peak": p_fp64, "unit": "FLOP/s",
                         "frac": fl2 / dt2 / p_fp64,
                         "flops": "of the method run (parity-class solve of mirror-symmetric cells)"},
            "reference_method_flops_per_s": fl2_ref / dt2}
        if with_cpu:
            try:
                out["cpu_baseline"] = rcwa_cpu_baseline(cells)
            except Exception as exc:
                out["cpu_baseline"] = {"unavailable": str(exc)[:200]}
    return out


def measure_inverse_design(steps=20, warmup=3, form=None):
    """Inverse-design step of the differentiation form: loss = -(encircled energy
    within 1 um) / (total) on the 70,688-pillar x 161^2 metalens, fills -> t by
    natural cubic splines over the 64-width RCWA library, gradient by the adjoint
    kernel behind torch.autograd, one Adam step (lr 1e-3). Times whole steps
    (forward FP64 field, adjoint, spline, optimizer) with CUDA events."""
    import torch

    from celeris_b200 import capi
    from celeris_b200 import torch_ops as T
    from celeris_b200.workloads import metalens_70k, rcwa_library_64

    ap, g = metalens_70k()
    cells = rcwa_library_64()
    res, info = capi.rcwa_batch([capi.rcwa_cell(**c) for c in cells])
    fill = np.array([c["fill_x"] for c in cells])
    t = np.array([res[2 * i]["tx0"] for i in range(len(cells))])
    spline = T.LibrarySpline(fill, np.abs(t), np.angle(t))
    grid = T.FarFieldGrid(g.n, g.half_window_um, g.z_um, ap.wavelength_um)
    dev = torch.device("cuda")
    px = torch.tensor(ap.px, device=dev)
    py = torch.tensor(ap.py, device=dev)
    w0 = np.random.default_rng(0).uniform(fill[1], fill[-2], ap.npil)
    w = torch.tensor(w0, device=dev, requires_grad=True)
    opt = torch.optim.Adam([w], lr=1e-3)

    form = capi.FORM_PLAIN_F64 if form is None else form

    def step():
        opt.zero_grad()
        L = T.encircled_energy_loss(T.rs_field(spline(w), px, py, grid, form), grid, 1.0)
        L.backward()
        opt.step()
        return L

    for _ in range(warmup):
        L0 = step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        L = step()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    terms = ap.npil * g.n * g.n
    return {"workload": "metalens_70k_161sq adjoint + Adam",
            "form": "f32c (precision forward + adjoint)" if form == capi.FORM_F32C else "plain FP64",
            "ms_per_step": ms, "steps": steps,
            "terms_per_s_fwd_plus_adjoint": 2 * terms / (ms * 1e-3),
            "loss_first": float(L0.detach()), "loss_last": float(L.detach())}


def measure_reference_gpu_kernel(ap, g, E64h, f32c_err, dev):
    """The reference's FP32 psf_kernel (src/celeris/cuda/propagate.cu:36-84),
    compiled unmodified for sm_100a into oracle/_ref, on this GPU: kernel-only
    terms/s and the error of its |E|^2 against the FP64 form, on the
    785,456-pillar x 1024^2 metalens and on the 70,688-pillar x 161^2 metalens,
    beside the same figures of the precision form; plus its public host-buffer
    call propagate_psf on the 70k metalens (per-call allocation and copies)."""
    import torch

    from celeris_b200 import capi
    from celeris_b200 import torch_ops as T
    from celeris_b200.workloads import metalens_70k
    from oracle import ref_cuda as RC

    if not RC.available():
        return {"unavailable": "oracle/_ref/libref_psf_cuda.so not built"}
    res = {"kernel": "psf_kernel (reference, FP32 throughout: sqrtf, sincosf(k R), 1/R)"}
    I64 = np.abs(E64h) ** 2
    RC.psf_kernel(ap.px, ap.py, ap.t, 0.0, 0.0, g.z_um, ap.k, 64, g.half_window_um, reps=1)  # warm-up
    I_ref, ms = RC.psf_kernel(ap.px, ap.py, ap.t, 0.0, 0.0, g.z_um, ap.k, g.n, g.half_window_um, reps=1)
    res["metalens_785k_1024sq"] = {
        "terms_per_s": ap.npil * g.npix / (ms * 1e-3), "kernel_ms": ms,
        "intensity_error_vs_fp64": float(np.max(np.abs(I_ref - I64)) / I64.max()),
        "field_error_vs_fp64_of_f32c": f32c_err}
    a0, g0 = metalens_70k()
    grid0 = T.FarFieldGrid(g0.n, g0.half_window_um, g0.z_um, a0.wavelength_um)
    px0, py0, t0_ = (torch.tensor(v, device=dev) for v in (a0.px, a0.py, a0.t))
    E64_0 = T.rs_field_dev(px0, py0, t0_, grid0, capi.FORM_PLAIN_F64).cpu().numpy()
    E32_0 = T.rs_field_dev(px0, py0, t0_, grid0, capi.FORM_F32C).cpu().numpy()
    I64_0 = np.abs(E64_0) ** 2
    RC.psf_kernel(a0.px, a0.py, a0.t, 0.0, 0.0, g0.z_um, a0.k, g0.n, g0.half_window_um, reps=2)
    I_ref0, ms0 = RC.psf_kernel(a0.px, a0.py, a0.t, 0.0, 0.0, g0.z_um, a0.k, g0.n, g0.half_window_um, reps=10)
    RC.propagate_psf(a0.px, a0.py, a0.t, 0.0, 0.0, g0.z_um, a0.k, g0.n, g0.half_window_um)
    t_api = []
    for _ in range(5):
        t1 = time.perf_counter()
        RC.propagate_psf(a0.px, a0.py, a0.t, 0.0, 0.0, g0.z_um, a0.k, g0.n, g0.half_window_um)
        t_api.append(time.perf_counter() - t1)
    res["metalens_70k_161sq"] = {
        "terms_per_s": a0.npil * g0.npix / (ms0 * 1e-3), "kernel_ms": ms0,
        "api_call_terms_per_s": a0.npil * g0.npix / float(np.median(t_api)),
        "intensity_error_vs_fp64": float(np.max(np.abs(I_ref0 - I64_0)) / I64_0.max()),
        "intensity_error_vs_fp64_of_f32c": float(np.max(np.abs(np.abs(E32_0) ** 2 - I64_0)) / I64_0.max()),
        "field_error_vs_fp64_of_f32c": float(np.max(np.abs(E32_0 - E64_0)) / np.max(np.abs(E64_0)))}
    return res


def run_gpu(args):
    import torch

    from celeris_b200 import capi
    from celeris_b200 import torch_ops as T

    world, rank, local = dist_init(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    ap, g, cy = workload(rank)
    grid = T.FarFieldGrid(g.n, g.half_window_um, g.z_um, ap.wavelength_um, 0.0, cy)
    px = torch.tensor(ap.px, device=dev)
    py = torch.tensor(ap.py, device=dev)
    t = torch.tensor(ap.t, device=dev)
    flush_buf = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def flush():
        flush_buf.zero_()

    capi.set_kernel_timing(True)
    f32 = lambda: T.rs_field_dev(px, py, t, grid, capi.FORM_F32C)  # noqa: E731
    for _ in range(args.warmup):
        f32()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = capi.launch_count()
    ms, kms = timed_steps(f32, args.steps, stream, flush)
    launches = capi.launch_count() - l0
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    total_ms = max_over_ranks(world, float(sum(ms)))
    terms = float(ap.npil) * g.npix
    value = terms * args.steps * world / (total_ms * 1e-3)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 terms, f64 k*z phase + chunk sums, TwoSum-compensated f32 tile sums",
        "data": "synthetic (seeded metalens aperture, default_rng(0))",
        "config": {"workload": WORKLOAD, "pillars": ap.npil, "grid": f"{g.n}x{g.n}",
                   "half_window_um": g.half_window_um, "z_um": g.z_um, "wavelength_um": ap.wavelength_um,
                   "form": "f32c", "sharding": "focal row blocks per rank, pillars replicated",
                   "l2": "flushed between timed steps (256 MiB write, outside the events)"},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if world > 1 and not args.quick:
        try:
            out["rcwa_sharded"] = measure_rcwa_sharded(world, rank)
        except Exception as exc:
            out["rcwa_sharded"] = {"unavailable": str(exc)[:200]}
    if rank != 0:
        return
    # ---- error of the chosen form against the FP64 form (full grid) ----------
    E32 = f32()
    E64 = T.rs_field_dev(px, py, t, grid, capi.FORM_PLAIN_F64)
    torch.cuda.synchronize()
    err = float((E32 - E64).abs().max() / E64.abs().max())
    out["error_vs_fp64"] = err
    # ---- roofline: dominant kernel = rs_f32c_kernel ---------------------------
    peaks = capi.probe_peaks()
    k_ms = float(np.mean(kms))
    achieved = terms / (k_ms * 1e-3)
    peak_mufu = peaks["mufu_per_s"] / 3.0      # rsqrt + sin + cos per term
    peak_fp32 = peaks["ffma_per_s"] * 2.0 / 28.0  # 28 FP32 flops per term as FMA pairs
    peak = min(peak_mufu, peak_fp32)
    out["roofline"] = {
        "kernel": "rs_f32c_kernel", "bound": "sfu" if peak_mufu <= peak_fp32 else "fp32",
        "achieved": achieved, "peak": peak, "unit": "terms/s", "frac": achieved / peak,
        "traffic": profiles_traffic("rs_f32c_kernel_metalens_785k"),
        "peak_source": "in-run probe kernels (MUFU sin.approx and FP32 FMA throughput on this GPU)",
        "measured_peaks": peaks, "kernel_ms_per_launch": k_ms,
        "algorithmic_bytes_per_launch": ap.npil * 16 + g.npix * 16,
    }
    # the HBM roof against the driver-measured copy bandwidth, for reference: far
    # below the binding SFU roof (the kernel reads each pillar tile once per CTA)
    hbm, src = measured_hbm_gbs()
    alg_gbs = (ap.npil * 16 + g.npix * 16) / (k_ms * 1e-3) / 1e9
    out["roofline"]["hbm"] = {"bound": "hbm", "achieved": alg_gbs, "peak": hbm, "unit": "GB/s",
                              "frac": alg_gbs / hbm, "traffic": out["roofline"]["traffic"], "peak_source": src}
    # ---- plain FP64 form, same workload ----------------------------------------
    f64 = lambda: T.rs_field_dev(px, py, t, grid, capi.FORM_PLAIN_F64)  # noqa: E731
    f64()
    ms64, kms64 = timed_steps(f64, 1 if args.quick else 2, stream, flush)
    v64 = terms / (np.mean(ms64) * 1e-3)
    out["plain_f64"] = {"value": v64, "unit": UNIT, "ms_per_step": float(np.mean(ms64)),
                        "roofline_frac_dfma": (terms / (np.mean(kms64) * 1e-3)) / (peaks["dfma_per_s"] * 2 / 21),
                        "chosen_over_plain": value / v64}
    # ---- the 70,688-pillar x 161^2 metalens, both forms ------------------------
    if not args.quick:
        from celeris_b200.workloads import metalens_70k

        a0, g0 = metalens_70k()
        grid0 = T.FarFieldGrid(g0.n, g0.half_window_um, g0.z_um, a0.wavelength_um)
        px0, py0, t0_ = (torch.tensor(v, device=dev) for v in (a0.px, a0.py, a0.t))
        res = {}
        for name, form in (("f32c", capi.FORM_F32C), ("plain_f64", capi.FORM_PLAIN_F64)):
            fn = lambda form=form: T.rs_field_dev(px0, py0, t0_, grid0, form)  # noqa: E731
            for _ in range(3):
                fn()
            m, km = timed_steps(fn, 10, stream, flush)
            res[name] = {"value": a0.npil * g0.npix / (np.mean(m) * 1e-3), "ms_per_step": float(np.mean(m)),
                         "kernel_ms": float(np.mean(km))}
        Ea = T.rs_field_dev(px0, py0, t0_, grid0, capi.FORM_F32C)
        Eb = T.rs_field_dev(px0, py0, t0_, grid0, capi.FORM_PLAIN_F64)
        res["f32c"]["error_vs_fp64"] = float((Ea - Eb).abs().max() / Eb.abs().max())
        out["metalens_70k_161sq"] = res
    # ---- e2e: the C-ABI host-buffer call ----------------------------------------
    E_host = None
    for _ in range(2):
        E_host, _, _, _ = capi.rs_field_bounded(ap.px, ap.py, ap.t, 0.0, cy, g.z_um, ap.k, g.n, g.half_window_um)
    e2e_t = []
    stated = bound = None
    for _ in range(args.steps):
        flush()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E_host, _, stated, bound = capi.rs_field_bounded(ap.px, ap.py, ap.t, 0.0, cy, g.z_um, ap.k, g.n,
                                                         g.half_window_um)
        e2e_t.append(time.perf_counter() - t0)
    # the true full-grid error of the returned field against the FP64 form
    E64h = E64.cpu().numpy()
    true_err = float(np.max(np.abs(E_host - E64h)) / np.max(np.abs(E_host)))
    out["e2e"] = {"value": terms / float(np.mean(e2e_t)), "unit": UNIT,
                  "h2d_bytes_per_step": int(ap.npil * 32), "d2h_bytes_per_step": int(g.npix * 16),
                  "api": "celeris_rs_field_bounded (C ABI, host buffers, F32C form, sampled error and bound stated)",
                  "stated_error": stated, "stated_bound": bound, "error_vs_fp64_full_grid": true_err,
                  "ms_per_step": 1e3 * float(np.mean(e2e_t))}
    # ---- the reference's own FP32 CUDA kernel (psf_kernel), unmodified ----------------
    if not args.quick:
        try:
            out["reference_gpu_kernel"] = measure_reference_gpu_kernel(ap, g, E64h, float(err), dev)
        except Exception as exc:
            out["reference_gpu_kernel"] = {"unavailable": str(exc)[:200]}
    # ---- RCWA cells/s ------------------------------------------------------------
    if not args.quick:
        try:
            out["inverse_design"] = measure_inverse_design()
            out["inverse_design_f32c"] = measure_inverse_design(form=capi.FORM_F32C)
        except Exception as exc:
            out["inverse_design"] = {"unavailable": str(exc)[:200]}
    rclk = ClockSampler(local)
    out["rcwa"] = measure_rcwa(peaks, quick=args.quick, with_cpu=not args.no_cpu, sampler=rclk)
    out["rcwa"]["clocks"] = rclk.stop()
    # ---- CPU baseline: the reference's own far-field on this host --------------
    if not args.no_cpu:
        try:
            out["cpu_baseline"] = cpu_reference_sample(ap, g)
        except Exception as exc:
            out["cpu_baseline"] = {"unavailable": str(exc)[:200]}
    print(json.dumps(out), flush=True)


def run_case(name, reps):
    """Run one named small case `reps` times (for ncu captures)."""
    import torch

    from celeris_b200 import capi
    from celeris_b200 import torch_ops as T
    from celeris_b200.workloads import metalens_70k, metalens_785k

    dev = torch.device("cuda")
    if name.startswith("rcwa"):
        # rcwa_library: the 64-cell library sweep; rcwa_M<m>_<ncell>: uneven-batch
        # cells of one harmonic count
        from celeris_b200.workloads import rcwa_library_64, rcwa_uneven_4096

        if name == "rcwa_library":
            cells = rcwa_library_64()
        else:
            _, m, nc = name.split("_")
            cells = [c for c in rcwa_uneven_4096() if c["Mx"] == int(m[1:])][: int(nc)]
        for _ in range(reps):
            capi.rcwa_batch([capi.rcwa_cell(**c) for c in cells])
        print(json.dumps({"case": name, "reps": reps, "cells": len(cells)}))
        return
    if name.startswith("ff785k"):
        ap, g = metalens_785k()
        n = int(name.split("_")[2]) if name.count("_") >= 2 else 256
        grid = T.FarFieldGrid(n, g.half_window_um, g.z_um, ap.wavelength_um)
    else:
        ap, g = metalens_70k()
        grid = T.FarFieldGrid(g.n, g.half_window_um, g.z_um, ap.wavelength_um)
    form = capi.FORM_PLAIN_F64 if "_f64" in name else capi.FORM_F32C
    px, py, t = (torch.tensor(v, device=dev) for v in (ap.px, ap.py, ap.t))
    for _ in range(reps):
        if "_adj" in name:
            v = torch.ones((grid.n, grid.n), dtype=torch.complex128, device=dev)
            T.rs_adjoint_dev(px, py, v, grid)
        else:
            T.rs_field_dev(px, py, t, grid, form)
    torch.cuda.synchronize()
    print(json.dumps({"case": name, "reps": reps, "pillars": ap.npil, "grid": grid.n}))


def main():
    args = parse()
    if args.case:
        run_case(args.case, args.reps)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    run_gpu(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
