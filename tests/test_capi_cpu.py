"""CPU checks of the C ABI: the library loads, exports every declared symbol,
and reports argument errors and the missing device with the documented codes
(no compute is attempted without a GPU)."""
import os
import re
import subprocess

import pytest

from celeris_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    hdr = open(os.path.join(ROOT, "include", "celeris_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(celeris_[a-z0-9_]+)\s*\(", hdr)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(capi.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (celeris_[a-z0-9_]+)$", out, flags=re.M))
    assert set(declared_functions()) <= exported


def test_abi_version_and_launch_counter():
    lib = capi.load()
    assert lib.celeris_abi_version() >= 10000
    assert capi.launch_count() >= 0


@pytest.mark.skipif(capi.load().celeris_available() != 0, reason="a device is present")
def test_no_device_is_an_error_not_a_fallback():
    import numpy as np

    with pytest.raises(capi.CelerisError) as e:
        capi.propagate_psf(np.zeros(3), np.zeros(3), np.ones(3, complex), 0, 0, 10.0, 1.0, 5, 1.0)
    assert e.value.status == capi.ERR_NO_DEVICE


def test_invalid_arguments_are_rejected_before_device_work():
    import numpy as np

    with pytest.raises(capi.CelerisError) as e:
        capi.rs_field(np.zeros(3), np.zeros(3), np.ones(3, complex), 0, 0, 10.0, 1.0, 5, 1.0, form=7)
    assert e.value.status == capi.ERR_INVALID_ARG
    lib = capi.load()
    st = lib.celeris_propagate_zx(None, None, None, 0, 0.0, 1.0, 1, 0.0, 1.0, 5, 1.0, None)
    assert st == capi.ERR_INVALID_ARG
    assert b"nx" in lib.celeris_last_error()


def test_stack_arguments_are_rejected_before_device_work():
    """Multi-layer stack entry points: layers that disagree on what the
    reference's Rcwa2DStack holds once (orders, periods, wavelength, angles,
    half-spaces), empty stacks, bad offsets and short order buffers are
    argument errors, reported without touching a device."""
    base = dict(period_um=0.4, wavelength_um=0.633, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0,
                fill_x=0.5, thickness_um=0.3, Mx=2)
    a = capi.rcwa_cell(**base)
    for change in (dict(period_um=0.5), dict(wavelength_um=0.6), dict(Mx=3), dict(n_sub=1.5),
                   dict(theta_rad=0.1)):
        b = capi.rcwa_cell(**{**base, **change})
        with pytest.raises(capi.CelerisError) as e:
            capi.solve_rcwa_2d_stack([a, b])
        assert e.value.status == capi.ERR_INVALID_ARG
        with pytest.raises(capi.CelerisError) as e:
            capi.rcwa_stack_batch([[a], [a, b]])
        assert e.value.status == capi.ERR_INVALID_ARG
    with pytest.raises(capi.CelerisError) as e:
        capi.rcwa_stack_batch([[a], []])
    assert e.value.status == capi.ERR_INVALID_ARG
    lib = capi.load()
    import ctypes

    arr = (capi.RcwaCell * 1)(a)
    out = capi.RcwaResult()
    orders = (capi.RcwaOrder * 4)()
    ex = (ctypes.c_double * 2)(1.0, 0.0)
    ey = (ctypes.c_double * 2)(0.0, 0.0)
    st = lib.celeris_solve_rcwa_2d_orders(arr, 1, ex, ey, ctypes.byref(out), orders, 4)  # 25 orders needed
    assert st == capi.ERR_INVALID_ARG and b"orders" in lib.celeris_last_error()
    assert lib.celeris_solve_rcwa_2d_stack(arr, 0, ex, ey, ctypes.byref(out)) == capi.ERR_INVALID_ARG


def test_eig_arguments_are_rejected_before_device_work():
    import numpy as np

    lib = capi.load()
    buf = np.zeros(8)
    assert lib.celeris_eig_general_batch(capi._dp(buf), 0, 1, capi._dp(buf), capi._dp(buf), None) == \
        capi.ERR_INVALID_ARG
    assert lib.celeris_eig_general_batch(capi._dp(buf), 5000, 1, capi._dp(buf), capi._dp(buf), None) == \
        capi.ERR_TOO_LARGE
    assert lib.celeris_eig_general(None, 4, capi._dp(buf), capi._dp(buf)) == capi.ERR_INVALID_ARG


def test_non_finite_rcwa_and_eig_inputs_are_rejected_before_device_work():
    """A NaN or Inf in any real field of a cell, or in a matrix handed to the
    eigensolver, is an argument error naming the cell / matrix, reported
    without touching a device (the reference would carry it into Eigen and
    return non-finite t, R, T)."""
    import math

    import numpy as np

    base = dict(period_um=0.4, wavelength_um=0.633, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0,
                fill_x=0.5, thickness_um=0.3, Mx=2)
    for key, bad in (("fill_x", math.nan), ("thickness_um", math.inf), ("eps_pillar", complex(4.0, math.nan)),
                     ("wavelength_um", math.inf), ("rotation_rad", -math.inf)):
        cells = [capi.rcwa_cell(**base), capi.rcwa_cell(**{**base, key: bad})]
        with pytest.raises(capi.CelerisError) as e:
            capi.rcwa_batch(cells)
        assert e.value.status == capi.ERR_INVALID_ARG, key
        assert "cell 1" in str(e.value)
    lib = capi.load()
    A = np.eye(6, dtype=complex)
    A2 = np.stack([A, A])
    A2[1, 2, 3] = complex(0.0, math.nan)
    out = np.zeros(2 * 2 * 36)
    assert lib.celeris_eig_general_batch(capi._dp(A2.view(np.float64)), 6, 2, capi._dp(out), capi._dp(out), None) \
        == capi.ERR_INVALID_ARG
    assert b"matrix 1" in lib.celeris_last_error()
