"""Failure detection on the GPU, without faulting it.

The reference degrades silently: propagate_psf returns false and the caller
falls back to its CPU loop (src/celeris/cuda/propagate.cu:137-139), a failed
zgeev falls back to Eigen (src/celeris/rcwa/eig.cpp:73-77). Here every failure
is a status code, and these tests drive each one from the host or through a
bounded device wait, then check that the device stays usable:
  - a bounded device wait that runs out  -> CELERIS_ERR_DEVICE_TIMEOUT
  - a device allocation that fails        -> CELERIS_ERR_OOM, nothing leaked
  - a QR eigensolve that hits its cap     -> CELERIS_ERR_EIG_NOCONV, per-cell info
  - NaN / Inf in the far-field inputs     -> CELERIS_ERR_INVALID_ARG on that stream
"""
import ctypes
import math
import threading

import numpy as np
import pytest

from celeris_b200 import capi
from celeris_b200.workloads import small_aperture
from oracle import farfield as F

pytestmark = pytest.mark.gpu


def _field_ok():
    a = small_aperture(300, seed=2)
    Eo = F.rs_field(a.px, a.py, a.t, 0.0, 0.0, a.focal_um, a.k, 17, 2.0)
    E, _, _ = capi.rs_field(a.px, a.py, a.t, 0.0, 0.0, a.focal_um, a.k, 17, 2.0)
    assert np.max(np.abs(E - Eo)) <= 1e-10 * np.max(np.abs(Eo))


def test_bounded_device_wait_reports_timeout_and_context_survives():
    lib = capi.load()
    for polls in (1, 1000):
        assert lib.celeris_device_wait_selftest(polls) == capi.ERR_DEVICE_TIMEOUT
        assert b"bounded device wait" in lib.celeris_last_error()
    _field_ok()


def _in_fresh_thread(fn):
    out = {}

    def run():
        out["v"] = fn()

    th = threading.Thread(target=run)
    th.start()
    th.join()
    return out["v"]


def test_injected_allocation_failure_is_oom_without_leak():
    import torch

    lib = capi.load()
    a = small_aperture(513, seed=4)

    def failing_host_call():
        # host-buffer call on a new thread: its device I/O buffer is the first allocation
        assert lib.celeris_debug_fail_alloc(1) == capi.OK
        return _in_fresh_thread(lambda: lib.celeris_propagate_psf(
            capi._dp(a.px), capi._dp(a.py), capi._dp(a.t.view(np.float64)), a.npil, 0.0, 0.0, a.focal_um, a.k, 9,
            1.0, capi._dp(np.zeros(81))))

    # the first thread of this kind also sets up the CUDA runtime's own per-thread
    # state; the second failing call must leave device memory exactly as it found it
    assert failing_host_call() == capi.ERR_OOM
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert failing_host_call() == capi.ERR_OOM
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # device-buffer call on a stream this library has not seen: its workspace arena
    dev = torch.device("cuda")
    px, py, t = (torch.tensor(v, device=dev) for v in (a.px, a.py, a.t))
    E = torch.empty((9, 9), dtype=torch.complex128, device=dev)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert lib.celeris_debug_fail_alloc(1) == capi.OK
    st = lib.celeris_rs_field_dev(capi.FORM_PLAIN_F64, ctypes.c_void_p(px.data_ptr()), ctypes.c_void_p(py.data_ptr()),
                                  ctypes.c_void_p(t.data_ptr()), a.npil, 0.0, 0.0, a.focal_um, a.k, 9, 1.0,
                                  ctypes.c_void_p(E.data_ptr()), None, ctypes.c_void_p(s.cuda_stream))
    assert st == capi.ERR_OOM
    assert b"injected" in lib.celeris_last_error()
    assert torch.cuda.mem_get_info()[0] == free1
    # the count is spent: the same call now succeeds
    assert lib.celeris_rs_field_dev(capi.FORM_PLAIN_F64, ctypes.c_void_p(px.data_ptr()),
                                    ctypes.c_void_p(py.data_ptr()), ctypes.c_void_p(t.data_ptr()), a.npil, 0.0, 0.0,
                                    a.focal_um, a.k, 9, 1.0, ctypes.c_void_p(E.data_ptr()), None,
                                    ctypes.c_void_p(s.cuda_stream)) == capi.OK
    assert lib.celeris_sync_status(ctypes.c_void_p(s.cuda_stream)) == capi.OK
    lib.celeris_debug_fail_alloc(0)
    _field_ok()


def test_injected_allocation_failure_in_an_rcwa_batch():
    lib = capi.load()
    cells = [capi.rcwa_cell(period_um=0.4, wavelength_um=0.633, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0,
                            fill_x=0.2 + 0.1 * i, thickness_um=0.6, Mx=2) for i in range(5)]
    ref, _ = capi.rcwa_batch(cells)

    def batch():
        arr = (capi.RcwaCell * len(cells))(*cells)
        out = (capi.RcwaResult * (2 * len(cells)))()
        return lib.celeris_rcwa_batch(arr, len(cells), out, None)

    assert lib.celeris_debug_fail_alloc(1) == capi.OK
    assert _in_fresh_thread(batch) == capi.ERR_OOM
    lib.celeris_debug_fail_alloc(0)
    got, info = capi.rcwa_batch(cells)
    assert np.all(info == 0)
    for a, b in zip(got, ref):
        assert a["tx0"] == b["tx0"]


def test_qr_iteration_cap_reports_non_convergence_per_cell():
    lib = capi.load()
    cells = [capi.rcwa_cell(period_um=0.4, wavelength_um=0.633, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0,
                            fill_x=0.3 + 0.1 * i, thickness_um=0.6, Mx=3) for i in range(4)]
    ref, _ = capi.rcwa_batch(cells)
    try:
        assert lib.celeris_debug_qr_iteration_cap(1) == capi.OK
        _, info = capi.rcwa_batch(cells)
        assert np.all(info > 0)  # LAPACK-style: 1 + index of the last unconverged eigenvalue
        assert np.all(info <= 98)
        arr = (capi.RcwaCell * len(cells))(*cells)
        out = (capi.RcwaResult * (2 * len(cells)))()
        assert lib.celeris_rcwa_batch(arr, len(cells), out, None) == capi.ERR_EIG_NOCONV
        msg = lib.celeris_last_error()
        assert b"cell 0" in msg and b"info" in msg
        rng = np.random.default_rng(1)
        A = rng.standard_normal((2, 60, 60)) + 1j * rng.standard_normal((2, 60, 60))
        Af = np.ascontiguousarray(np.transpose(A, (0, 2, 1)))
        ev, vec = np.empty((2, 60), complex), np.empty((2, 60, 60), complex)
        inf = np.zeros(2, dtype=np.int32)
        assert lib.celeris_eig_general_batch(capi._dp(Af.view(np.float64)), 60, 2, capi._dp(ev.view(np.float64)),
                                             capi._dp(vec.view(np.float64)),
                                             inf.ctypes.data_as(ctypes.POINTER(ctypes.c_int))) == capi.OK
        assert np.all(inf > 0)
    finally:
        lib.celeris_debug_qr_iteration_cap(0)
    got, info = capi.rcwa_batch(cells)
    assert np.all(info == 0)
    for a, b in zip(got, ref):
        assert abs(a["tx0"] - b["tx0"]) <= 1e-13 * abs(b["tx0"])


def test_non_finite_far_field_inputs_are_reported_on_their_stream():
    import torch

    lib = capi.load()
    a = small_aperture(700, seed=9)
    for bad in (math.nan, math.inf):
        px = a.px.copy()
        px[123] = bad
        with pytest.raises(capi.CelerisError) as ei:
            capi.rs_field(px, a.py, a.t, 0.0, 0.0, a.focal_um, a.k, 11, 1.0, form=capi.FORM_F32C)
        assert ei.value.status == capi.ERR_INVALID_ARG
        assert "NaN or Inf" in str(ei.value)
    # device form: the flag stays with the stream that ran the call
    dev = torch.device("cuda")
    t = torch.tensor(a.t, device=dev)
    t[5] = complex(math.nan, 0.0)
    px, py = torch.tensor(a.px, device=dev), torch.tensor(a.py, device=dev)
    E = torch.empty((11, 11), dtype=torch.complex128, device=dev)
    s_bad, s_other = torch.cuda.Stream(), torch.cuda.Stream()
    assert lib.celeris_rs_field_dev(capi.FORM_PLAIN_F64, ctypes.c_void_p(px.data_ptr()),
                                    ctypes.c_void_p(py.data_ptr()), ctypes.c_void_p(t.data_ptr()), a.npil, 0.0, 0.0,
                                    a.focal_um, a.k, 11, 1.0, ctypes.c_void_p(E.data_ptr()), None,
                                    ctypes.c_void_p(s_bad.cuda_stream)) == capi.OK
    assert lib.celeris_sync_status(ctypes.c_void_p(s_other.cuda_stream)) == capi.OK
    assert lib.celeris_sync_status(ctypes.c_void_p(s_bad.cuda_stream)) == capi.ERR_INVALID_ARG
    assert lib.celeris_sync_status(ctypes.c_void_p(s_bad.cuda_stream)) == capi.OK  # read once, then cleared
    assert torch.isnan(E).any()
    _field_ok()
