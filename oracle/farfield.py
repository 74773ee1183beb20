"""ORACLE - test infrastructure only.

ctypes access to the far-field checkers built by oracle/Makefile:
  * liboracle_ff.so   - the plain-C restatement (farfield_oracle.c) of the
                        reference loops in src/celeris/analysis/focal.cpp:223-236
                        and throughfocus.cpp:105-118, returning the complex field;
  * libref_farfield.so - the reference's own CPU propagate_pillars
                        (focal.cpp:205-238), compiled from its sources.
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
module, as the checker; the product path never imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_P = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)
_D = ctypes.c_double
_lib = None
_ref = None


def _dp(a):
    return a.ctypes.data_as(_P)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "_build", "liboracle_ff.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        _lib = ctypes.CDLL(path)
    return _lib


def ref_lib():
    """The reference's own CPU far-field, or None when it was not built."""
    global _ref
    if _ref is None:
        path = os.path.join(_HERE, "_ref", "libref_farfield.so")
        if not os.path.exists(path):
            return None
        _ref = ctypes.CDLL(path)
        _ref.ref_hardware_threads.restype = ctypes.c_int
    return _ref


def _c128(t):
    return np.ascontiguousarray(t, dtype=np.complex128)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def rs_field(px, py, t, cx, cy, z, k, n, half_window, rows=None):
    """Complex field E (n x n, complex128) of the RS sum; rows=(lo, hi) limits
    the evaluated rows (other rows stay 0)."""
    px, py, t = _f64(px), _f64(py), _c128(t)
    out = np.zeros((n, n), dtype=np.complex128)
    lo, hi = (0, n) if rows is None else rows
    lib().rs_field(_dp(px), _dp(py), _dp(t.view(np.float64)), ctypes.c_int(len(px)), _D(cx), _D(cy),
                   _D(z), _D(k), ctypes.c_int(n), _D(half_window), ctypes.c_int(lo), ctypes.c_int(hi),
                   _dp(out.view(np.float64)), None)
    return out


def rs_pixels(px, py, t, cx, cy, z, k, n, half_window, idx):
    px, py, t = _f64(px), _f64(py), _c128(t)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    out = np.zeros(len(idx), dtype=np.complex128)
    lib().rs_pixels(_dp(px), _dp(py), _dp(t.view(np.float64)), ctypes.c_int(len(px)), _D(cx), _D(cy),
                    _D(z), _D(k), ctypes.c_int(n), _D(half_window), idx.ctypes.data_as(_PI),
                    ctypes.c_int(len(idx)), _dp(out.view(np.float64)))
    return out


def rs_zx(px, py, t, xmin, xmax, nx, zmin, zmax, nz, k):
    px, py, t = _f64(px), _f64(py), _c128(t)
    out = np.zeros((nz, nx), dtype=np.float64)
    lib().rs_zx(_dp(px), _dp(py), _dp(t.view(np.float64)), ctypes.c_int(len(px)), _D(xmin), _D(xmax),
                ctypes.c_int(nx), _D(zmin), _D(zmax), ctypes.c_int(nz), _D(k), _dp(out))
    return out


def rs_adjoint(px, py, cx, cy, z, k, n, half_window, v):
    px, py = _f64(px), _f64(py)
    v = _c128(v).reshape(-1)
    out = np.zeros(len(px), dtype=np.complex128)
    lib().rs_adjoint(_dp(px), _dp(py), ctypes.c_int(len(px)), _D(cx), _D(cy), _D(z), _D(k),
                     ctypes.c_int(n), _D(half_window), _dp(v.view(np.float64)), _dp(out.view(np.float64)))
    return out


def ref_propagate_pillars(px, py, t, cx, cy, z, wavelength_um, n, half_window):
    """|E|^2 from the reference's own celeris::propagate_pillars (CPU FP64)."""
    r = ref_lib()
    if r is None:
        raise FileNotFoundError("oracle/_ref/libref_farfield.so not built")
    px, py, t = _f64(px), _f64(py), _c128(t)
    out = np.zeros((n, n), dtype=np.float64)
    r.ref_propagate_pillars(_dp(px), _dp(py), _dp(t.view(np.float64)), ctypes.c_int(len(px)), _D(cx),
                            _D(cy), _D(z), _D(wavelength_um), ctypes.c_int(n), _D(half_window), _dp(out))
    return out


def ref_threads():
    r = ref_lib()
    return None if r is None else int(r.ref_hardware_threads())


# ---- the reference's own analyses (field.cpp, throughfocus.cpp) on a lens given
# as arrays: n_cells, period, fill_map [n_cells^2], library fill/phase/amplitude.
def _lens_args(lens_n, period, fill_map, lib_fill, lib_phase, lib_amp, lib_wl):
    fm, lf, lp, la = (_f64(np.ravel(a)) for a in (fill_map, lib_fill, lib_phase, lib_amp))
    keep = (fm, lf, lp, la)
    args = [ctypes.c_int(lens_n), _D(period), _dp(fm), ctypes.c_int(len(lf)), _dp(lf), _dp(lp), _dp(la), _D(lib_wl)]
    return args, keep


def _ref_or_raise():
    r = ref_lib()
    if r is None:
        raise FileNotFoundError("oracle/_ref/libref_farfield.so not built")
    return r


def ref_through_focus(lens_args, f, wl, D):
    """celeris::analyze_through_focus (throughfocus.cpp:15-78, CPU): z, normalized
    on-axis intensity, z_peak, depth of focus."""
    r = _ref_or_raise()
    args, keep = _lens_args(*lens_args)
    z = np.zeros(161, dtype=np.float32)
    I = np.zeros(161, dtype=np.float32)
    sc = np.zeros(2)
    fp = ctypes.POINTER(ctypes.c_float)
    r.ref_through_focus(*args, _D(f), _D(wl), _D(D), z.ctypes.data_as(fp), I.ctypes.data_as(fp), _dp(sc))
    return z, I, sc[0], sc[1]


def ref_field_of_view(lens_args, f, wl, D, angles):
    r = _ref_or_raise()
    args, keep = _lens_args(*lens_args)
    a = _f64(angles)
    out = np.zeros((len(a), 3))
    r.ref_field_of_view(*args, _D(f), _D(wl), _D(D), _dp(a), ctypes.c_int(len(a)), _dp(out))
    return out


def ref_wide_fov(lens_args, f, wl, D_lens, D_stop, stop_dist, angles):
    r = _ref_or_raise()
    args, keep = _lens_args(*lens_args)
    a = _f64(angles)
    out = np.zeros((len(a), 3))
    r.ref_wide_fov(*args, _D(f), _D(wl), _D(D_lens), _D(D_stop), _D(stop_dist), _dp(a), ctypes.c_int(len(a)),
                   _dp(out))
    return out


def ref_field_grid(lens_args, f, wl, D, max_angle, n_half, psf_n):
    r = _ref_or_raise()
    args, keep = _lens_args(*lens_args)
    n = 2 * n_half + 1
    out = np.zeros((n * n, 7))
    r.ref_field_grid(*args, _D(f), _D(wl), _D(D), _D(max_angle), ctypes.c_int(n_half), ctypes.c_int(psf_n),
                     _dp(out))
    return out


def ref_chromatic(lens_args, f, wl, D, lam_min, lam_max, n):
    """celeris::analyze_chromatic (chromatic.cpp, CPU): rows (lambda, focal z, rel_peak)."""
    r = _ref_or_raise()
    args, keep = _lens_args(*lens_args)
    out = np.zeros((n, 3))
    r.ref_chromatic(*args, _D(f), _D(wl), _D(D), _D(lam_min), _D(lam_max), ctypes.c_int(n), _dp(out))
    return out


def ref_tolerance(lens_args, f, wl, D, sigmas, trials, seed):
    """celeris::analyze_tolerance (tolerance.cpp, CPU): rows (sigma, mean, std, worst Strehl)."""
    r = _ref_or_raise()
    args, keep = _lens_args(*lens_args)
    sg = _f64(sigmas)
    out = np.zeros((len(sigmas), 4))
    r.ref_tolerance(*args, _D(f), _D(wl), _D(D), _dp(sg), ctypes.c_int(len(sigmas)), ctypes.c_int(trials),
                    ctypes.c_uint(seed), _dp(out))
    return out
