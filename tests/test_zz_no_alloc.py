"""The far-field entry point that allocates nothing (celeris_rs_field_noalloc).

Some callers cannot let a library allocate device memory (their pool owns the
GPU's free memory, or they cannot afford the device-wide synchronisation of
cudaMalloc/cudaFree). This entry point keeps its scratch in a fixed 48 MiB
array inside the library. These tests call it through the C ABI with device
buffers and compare two calls in a row with the allocating entry point
celeris_rs_field_dev, at the tolerances of the far-field tests (plain FP64
1e-10, FP32-compensated 1e-5, relative to the peak |E|). The file is named so
pytest collects it last; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from celeris_b200 import capi
from celeris_b200.workloads import metalens_70k, small_aperture

pytestmark = pytest.mark.gpu

TOL = {capi.FORM_PLAIN_F64: 1e-10, capi.FORM_F32C: 1e-5}


def _run(fn, form, px, py, t, cx, cy, z, k, n, W):
    import torch

    E = torch.full((n, n), complex("nan"), dtype=torch.complex128, device="cuda")
    I = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    capi.check(fn(form, ctypes.c_void_p(px.data_ptr()), ctypes.c_void_p(py.data_ptr()),
                  ctypes.c_void_p(t.data_ptr()), int(px.numel()), cx, cy, z, k, n, W,
                  ctypes.c_void_p(E.data_ptr()), ctypes.c_void_p(I.data_ptr()), st))
    torch.cuda.synchronize()
    return E.cpu().numpy(), I.cpu().numpy()


@pytest.mark.parametrize("form", [capi.FORM_PLAIN_F64, capi.FORM_F32C], ids=["plain_f64", "f32c"])
@pytest.mark.parametrize("case", ["metalens_70k", "ragged_1025", "merged_chunks_20011"])
def test_noalloc_matches_allocating_entry_point_twice(form, case):
    import torch

    lib = capi.load()
    if case == "metalens_70k":
        ap, g = metalens_70k()
        args = (0.0, 0.0, g.z_um, ap.k, g.n, g.half_window_um)
    elif case == "ragged_1025":
        ap = small_aperture(1025, seed=7)
        args = (0.3, -0.2, ap.focal_um, ap.k, 37, 2.5)
    else:
        # 1024^2 pixels: one grid of partial sums is 16 MiB, so the precision
        # form's usual pillar split (six or more chunks) does not fit in the
        # 48 MiB scratch and the chunks are merged until it does
        ap = small_aperture(20011, seed=5, spread_um=30.0, focal_um=200.0)
        args = (0.0, 0.0, ap.focal_um, ap.k, 1024, 6.0)
    dev = torch.device("cuda")
    px, py, t = (torch.tensor(v, device=dev) for v in (ap.px, ap.py, ap.t))
    E_ref, I_ref = _run(lib.celeris_rs_field_dev, form, px, py, t, *args)
    peak = np.max(np.abs(E_ref))
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        E, I = _run(lib.celeris_rs_field_noalloc, form, px, py, t, *args)
        assert np.max(np.abs(E - E_ref)) <= TOL[form] * peak
        assert np.max(np.abs(I - I_ref)) <= 2.5 * TOL[form] * peak ** 2


def test_noalloc_rejects_requests_beyond_its_scratch():
    import torch

    lib = capi.load()
    ap = small_aperture(16, seed=3)
    dev = torch.device("cuda")
    px, py, t = (torch.tensor(v, device=dev) for v in (ap.px, ap.py, ap.t))
    n = 2000  # 4e6 pixels x 16 B of partial sums > 48 MiB
    E = torch.empty((n, n), dtype=torch.complex128, device=dev)
    st = lib.celeris_rs_field_noalloc(capi.FORM_F32C, ctypes.c_void_p(px.data_ptr()), ctypes.c_void_p(py.data_ptr()),
                                      ctypes.c_void_p(t.data_ptr()), 16, 0.0, 0.0, 30.0, ap.k, n, 2.0,
                                      ctypes.c_void_p(E.data_ptr()), None, None)
    assert st == capi.ERR_TOO_LARGE
    assert b"limit" in lib.celeris_last_error()


def test_noalloc_set_up_call_with_nothing_to_compute():
    """n = 0 (and no pillars) only sets up the scratch on the current device: the
    call a caller makes before its memory pool takes the free memory."""
    lib = capi.load()
    assert lib.celeris_rs_field_noalloc(capi.FORM_F32C, None, None, None, 0, 0.0, 0.0, 30.0, 10.0, 0, 1.0,
                                        None, None, None) == capi.OK
    assert lib.celeris_rs_field_noalloc(capi.FORM_PLAIN_F64, None, None, None, 0, 0.0, 0.0, 30.0, 10.0, 0, 1.0,
                                        None, None, None) == capi.OK
