"""ctypes binding of the C ABI in include/celeris_b200.h (libceleris_b200.so).

This is the reference-facing boundary as a Python caller (or a test) sees it:
plain pointers and sizes, int status codes turned into CelerisError. The
library is loaded from this package directory; a missing library raises
immediately (there is no CPU fallback anywhere in the product path).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libceleris_b200.so")

OK = 0
ERR_NO_DEVICE = 1
ERR_INVALID_ARG = 2
ERR_OOM = 3
ERR_CUDA = 4
ERR_EIG_NOCONV = 5
ERR_TOO_LARGE = 6
ERR_DEVICE_TIMEOUT = 7
ERR_SINGULAR = 8

FORM_PLAIN_F64 = 0
FORM_F32C = 1

SHAPE_RECT = 0
SHAPE_ELLIPSE = 1
SHAPE_CROSS = 2
SHAPE_RING = 3

_STATUS_NAMES = {
    ERR_NO_DEVICE: "no CUDA device",
    ERR_INVALID_ARG: "invalid argument",
    ERR_OOM: "out of memory",
    ERR_CUDA: "CUDA error",
    ERR_EIG_NOCONV: "eigensolve did not converge",
    ERR_TOO_LARGE: "size beyond limit",
    ERR_DEVICE_TIMEOUT: "device wait timed out",
    ERR_SINGULAR: "singular matrix",
}

# Every symbol the header declares (checked by the CPU test suite).
EXPORTED = [
    "celeris_available", "celeris_device_name", "celeris_last_error", "celeris_abi_version",
    "celeris_launch_count", "celeris_release_workspace", "celeris_propagate_psf",
    "celeris_propagate_zx", "celeris_rs_field", "celeris_rs_field_dev", "celeris_rs_adjoint_dev",
    "celeris_rs_check_dev", "celeris_sync_status", "celeris_solve_rcwa_2d", "celeris_rcwa_batch",
    "celeris_probe_peaks", "celeris_set_kernel_timing", "celeris_last_kernel_ms",
    "celeris_rs_field_noalloc", "celeris_rcwa_tuning_report",
    "celeris_probe_dmma", "celeris_solve_rcwa_2d_stack", "celeris_rcwa_stack_batch",
    "celeris_solve_rcwa_2d_orders", "celeris_eig_general", "celeris_eig_general_batch",
    "celeris_probe_mufu_accuracy", "celeris_rs_field_bounded", "celeris_rs_error_bound_dev",
    "celeris_rs_field_rows_dev", "celeris_rs_adjoint_rows_dev", "celeris_device_wait_selftest",
    "celeris_debug_fail_alloc", "celeris_debug_qr_iteration_cap",
]


class CelerisError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}: {_STATUS_NAMES.get(status, 'error')}] {msg}")
        self.status = status


class RcwaCell(ctypes.Structure):
    """celeris_rcwa_cell (include/celeris_b200.h)."""
    _fields_ = [
        ("period_x_um", ctypes.c_double), ("period_y_um", ctypes.c_double),
        ("wavelength_um", ctypes.c_double), ("theta_rad", ctypes.c_double), ("phi_rad", ctypes.c_double),
        ("n_inc", ctypes.c_double * 2), ("n_sub", ctypes.c_double * 2),
        ("eps_pillar", ctypes.c_double * 2), ("eps_bg", ctypes.c_double * 2),
        ("fill_x", ctypes.c_double), ("fill_y", ctypes.c_double), ("thickness_um", ctypes.c_double),
        ("shape_param", ctypes.c_double), ("rotation_rad", ctypes.c_double),
        ("shape", ctypes.c_int), ("Mx", ctypes.c_int), ("My", ctypes.c_int),
        ("grid", ctypes.c_int), ("force_laurent", ctypes.c_int),
    ]


class RcwaResult(ctypes.Structure):
    """celeris_rcwa_result (include/celeris_b200.h)."""
    _fields_ = [
        ("R", ctypes.c_double), ("T", ctypes.c_double), ("sum_de", ctypes.c_double),
        ("de_t0", ctypes.c_double), ("de_r0", ctypes.c_double),
        ("tx0", ctypes.c_double * 2), ("ty0", ctypes.c_double * 2),
    ]


class RcwaOrder(ctypes.Structure):
    """celeris_rcwa_order (include/celeris_b200.h)."""
    _fields_ = [
        ("p", ctypes.c_int), ("q", ctypes.c_int), ("de_t", ctypes.c_double), ("de_r", ctypes.c_double),
        ("prop_t", ctypes.c_int), ("prop_r", ctypes.c_int),
    ]


_lib = None
_P = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)
_D = ctypes.c_double
_I = ctypes.c_int
_V = ctypes.c_void_p


def load(path: str = LIB_PATH):
    """Load libceleris_b200.so and declare argument types. Raises when absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CelerisError(ERR_NO_DEVICE, f"{path} not built: run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    sig = {
        "celeris_available": (_I, []),
        "celeris_device_name": (ctypes.c_char_p, []),
        "celeris_last_error": (ctypes.c_char_p, []),
        "celeris_abi_version": (_I, []),
        "celeris_launch_count": (ctypes.c_uint64, []),
        "celeris_release_workspace": (_I, []),
        "celeris_propagate_psf": (_I, [_P, _P, _P, _I, _D, _D, _D, _D, _I, _D, _P]),
        "celeris_propagate_zx": (_I, [_P, _P, _P, _I, _D, _D, _I, _D, _D, _I, _D, _P]),
        "celeris_rs_field": (_I, [_I, _P, _P, _P, _I, _D, _D, _D, _D, _I, _D, _P, _P, _P]),
        "celeris_rs_field_dev": (_I, [_I, _V, _V, _V, _I, _D, _D, _D, _D, _I, _D, _V, _V, _V]),
        "celeris_rs_field_noalloc": (_I, [_I, _V, _V, _V, _I, _D, _D, _D, _D, _I, _D, _V, _V, _V]),
        "celeris_rs_adjoint_dev": (_I, [_I, _V, _V, _I, _D, _D, _D, _D, _I, _D, _V, _V, _V]),
        "celeris_rs_check_dev": (_I, [_V, _V, _V, _I, _D, _D, _D, _D, _I, _D, _V, _V, _I, _P, _V]),
        "celeris_sync_status": (_I, [_V]),
        "celeris_probe_peaks": (_I, [_P, _P, _P]),
        "celeris_probe_dmma": (_I, [_P]),
        "celeris_probe_mufu_accuracy": (_I, [_P, _P]),
        "celeris_rs_field_bounded": (_I, [_I, _P, _P, _P, _I, _D, _D, _D, _D, _I, _D, _P, _P, _P, _P]),
        "celeris_rs_error_bound_dev": (_I, [_V, _V, _V, _I, _D, _D, _D, _D, _I, _D, _V, _P, _V]),
        "celeris_rs_field_rows_dev": (_I, [_I, _V, _V, _V, _I, _D, _D, _D, _D, _I, _D, _I, _I, _V, _V, _V]),
        "celeris_rs_adjoint_rows_dev": (_I, [_I, _V, _V, _I, _D, _D, _D, _D, _I, _D, _I, _I, _V, _V, _V]),
        "celeris_device_wait_selftest": (_I, [ctypes.c_uint]),
        "celeris_debug_fail_alloc": (_I, [_I]),
        "celeris_debug_qr_iteration_cap": (_I, [_I]),
        "celeris_set_kernel_timing": (_I, [_I]),
        "celeris_last_kernel_ms": (_I, [_P]),
        "celeris_solve_rcwa_2d": (_I, [ctypes.POINTER(RcwaCell), _P, _P, ctypes.POINTER(RcwaResult)]),
        "celeris_rcwa_batch": (_I, [ctypes.POINTER(RcwaCell), _I, ctypes.POINTER(RcwaResult), _PI]),
        "celeris_rcwa_tuning_report": (_I, [ctypes.c_char_p, _I]),
        "celeris_solve_rcwa_2d_stack": (_I, [ctypes.POINTER(RcwaCell), _I, _P, _P, ctypes.POINTER(RcwaResult)]),
        "celeris_rcwa_stack_batch": (_I, [ctypes.POINTER(RcwaCell), _PI, _I, ctypes.POINTER(RcwaResult), _PI]),
        "celeris_eig_general": (_I, [_P, _I, _P, _P]),
        "celeris_eig_general_batch": (_I, [_P, _I, _I, _P, _P, _PI]),
        "celeris_solve_rcwa_2d_orders": (_I, [ctypes.POINTER(RcwaCell), _I, _P, _P, ctypes.POINTER(RcwaResult),
                                              ctypes.POINTER(RcwaOrder), _I]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int):
    if status != OK:
        msg = load().celeris_last_error().decode(errors="replace")
        raise CelerisError(status, msg)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def available() -> bool:
    return bool(load().celeris_available())


def device_name() -> str:
    return load().celeris_device_name().decode()


def launch_count() -> int:
    return int(load().celeris_launch_count())


def probe_peaks() -> dict:
    """Measured MUFU / FP32-FMA / FP64-FMA op rates of the current device."""
    a, b, c = (np.zeros(1) for _ in range(3))
    check(load().celeris_probe_peaks(_dp(a), _dp(b), _dp(c)))
    d = np.zeros(1)
    check(load().celeris_probe_dmma(_dp(d)))
    return {"mufu_per_s": float(a[0]), "ffma_per_s": float(b[0]), "dfma_per_s": float(c[0]),
            "dmma_fma_per_s": float(d[0])}


def set_kernel_timing(on: bool):
    check(load().celeris_set_kernel_timing(1 if on else 0))


def last_kernel_ms() -> float:
    v = np.zeros(1)
    check(load().celeris_last_kernel_ms(_dp(v)))
    return float(v[0])


def propagate_psf(px, py, pt, cx, cy, z, k, n, half_window) -> np.ndarray:
    """celeris::cuda::propagate_psf drop-in: |E|^2 (n x n) in the plain FP64 form."""
    px, py, pt = _f64(px), _f64(py), _c128(pt)
    out = np.empty((n, n), dtype=np.float64)
    check(load().celeris_propagate_psf(_dp(px), _dp(py), _dp(pt.view(np.float64)), len(px), cx, cy, z,
                                       k, n, half_window, _dp(out)))
    return out


def propagate_zx(px, py, pt, xmin, xmax, nx, zmin, zmax, nz, k) -> np.ndarray:
    px, py, pt = _f64(px), _f64(py), _c128(pt)
    out = np.empty((nz, nx), dtype=np.float64)
    check(load().celeris_propagate_zx(_dp(px), _dp(py), _dp(pt.view(np.float64)), len(px), xmin, xmax, nx,
                                      zmin, zmax, nz, k, _dp(out)))
    return out


def rs_field(px, py, pt, cx, cy, z, k, n, half_window, form=FORM_PLAIN_F64, want_field=True,
             want_intensity=True, want_err=False):
    """Far-field on host buffers. Returns (field complex128 | None, intensity | None, err)."""
    px, py, pt = _f64(px), _f64(py), _c128(pt)
    fld = np.empty((n, n), dtype=np.complex128) if want_field else None
    inten = np.empty((n, n), dtype=np.float64) if want_intensity else None
    err = np.zeros(1, dtype=np.float64)
    check(load().celeris_rs_field(form, _dp(px), _dp(py), _dp(pt.view(np.float64)), len(px), cx, cy, z, k,
                                  n, half_window, _dp(fld.view(np.float64)) if fld is not None else None,
                                  _dp(inten) if inten is not None else None,
                                  _dp(err) if want_err else None))
    return fld, inten, float(err[0])


def rs_field_bounded(px, py, pt, cx, cy, z, k, n, half_window, form=FORM_F32C, want_field=True,
                     want_intensity=False):
    """celeris_rs_field_bounded: (field | None, intensity | None, sampled error, error bound)."""
    px, py, pt = _f64(px), _f64(py), _c128(pt)
    fld = np.empty((n, n), dtype=np.complex128) if want_field else None
    inten = np.empty((n, n), dtype=np.float64) if want_intensity else None
    err = np.zeros(1, dtype=np.float64)
    bound = np.zeros(1, dtype=np.float64)
    check(load().celeris_rs_field_bounded(form, _dp(px), _dp(py), _dp(pt.view(np.float64)), len(px), cx, cy, z,
                                          k, n, half_window, _dp(fld.view(np.float64)) if fld is not None else None,
                                          _dp(inten) if inten is not None else None, _dp(err), _dp(bound)))
    return fld, inten, float(err[0]), float(bound[0])


def probe_mufu_accuracy() -> dict:
    """Measured (exhaustive) and assumed accuracy of sin/cos/rsqrt.approx."""
    m = np.zeros(3)
    a = np.zeros(3)
    check(load().celeris_probe_mufu_accuracy(_dp(m), _dp(a)))
    return {"measured": {"sin_abs": m[0], "cos_abs": m[1], "rsqrt_rel": m[2]},
            "model": {"sin_abs": a[0], "cos_abs": a[1], "rsqrt_rel": a[2]}}


def rcwa_cell(**kw) -> RcwaCell:
    c = RcwaCell()
    c.period_x_um = kw.get("period_x_um", kw.get("period_um", 0.4))
    c.period_y_um = kw.get("period_y_um", kw.get("period_um", 0.4))
    c.wavelength_um = kw["wavelength_um"]
    c.theta_rad = kw.get("theta_rad", 0.0)
    c.phi_rad = kw.get("phi_rad", 0.0)
    for name in ("n_inc", "n_sub", "eps_pillar", "eps_bg"):
        v = complex(kw[name])
        getattr(c, name)[0] = v.real
        getattr(c, name)[1] = v.imag
    c.fill_x = kw["fill_x"]
    c.fill_y = kw.get("fill_y", kw["fill_x"])
    c.thickness_um = kw["thickness_um"]
    c.shape_param = kw.get("shape_param", 0.5)
    c.rotation_rad = kw.get("rotation_rad", 0.0)
    c.shape = kw.get("shape", SHAPE_RECT)
    c.Mx = kw["Mx"]
    c.My = kw.get("My", kw["Mx"])
    c.grid = kw.get("grid", 0)
    c.force_laurent = kw.get("force_laurent", 0)
    return c


def result_dict(r: RcwaResult) -> dict:
    return {"R": r.R, "T": r.T, "sum_de": r.sum_de, "de_t0": r.de_t0, "de_r0": r.de_r0,
            "tx0": complex(r.tx0[0], r.tx0[1]), "ty0": complex(r.ty0[0], r.ty0[1])}


def solve_rcwa_2d(cell: RcwaCell, Ex0=1.0 + 0j, Ey0=0.0 + 0j) -> dict:
    ex = np.array([complex(Ex0).real, complex(Ex0).imag])
    ey = np.array([complex(Ey0).real, complex(Ey0).imag])
    out = RcwaResult()
    check(load().celeris_solve_rcwa_2d(ctypes.byref(cell), _dp(ex), _dp(ey), ctypes.byref(out)))
    return result_dict(out)


def rcwa_tuning_report() -> str:
    buf = ctypes.create_string_buffer(1 << 16)
    check(load().celeris_rcwa_tuning_report(buf, len(buf)))
    return buf.value.decode()


def rcwa_batch(cells) -> tuple[list[dict], np.ndarray]:
    """Batched cells; returns ([{X results}, {Y results}] per cell flattened, info)."""
    n = len(cells)
    arr = (RcwaCell * n)(*cells)
    out = (RcwaResult * (2 * n))()
    info = np.zeros(n, dtype=np.int32)
    check(load().celeris_rcwa_batch(arr, n, out, info.ctypes.data_as(_PI)))
    return [result_dict(out[i]) for i in range(2 * n)], info


def solve_rcwa_2d_stack(layers, Ex0=1.0 + 0j, Ey0=0.0 + 0j) -> dict:
    """Multi-layer stack (layers[0] next to the incident half-space)."""
    n = len(layers)
    arr = (RcwaCell * n)(*layers)
    ex = np.array([complex(Ex0).real, complex(Ex0).imag])
    ey = np.array([complex(Ey0).real, complex(Ey0).imag])
    out = RcwaResult()
    check(load().celeris_solve_rcwa_2d_stack(arr, n, _dp(ex), _dp(ey), ctypes.byref(out)))
    return result_dict(out)


def rcwa_stack_batch(stacks) -> tuple[list[dict], np.ndarray]:
    """Batched stacks (a list of layer lists); returns ([X, Y] results per stack flattened, info)."""
    flat = [c for st in stacks for c in st]
    start = np.zeros(len(stacks) + 1, dtype=np.int32)
    start[1:] = np.cumsum([len(st) for st in stacks])
    arr = (RcwaCell * max(len(flat), 1))(*flat)
    out = (RcwaResult * max(2 * len(stacks), 1))()
    info = np.zeros(max(len(stacks), 1), dtype=np.int32)
    check(load().celeris_rcwa_stack_batch(arr, start.ctypes.data_as(_PI), len(stacks), out,
                                          info.ctypes.data_as(_PI)))
    return [result_dict(out[i]) for i in range(2 * len(stacks))], info[:len(stacks)]


def solve_rcwa_2d_orders(layers, Ex0=1.0 + 0j, Ey0=0.0 + 0j) -> tuple[dict, list[dict]]:
    """One stack (one layer or several) with the per-order efficiencies."""
    n = len(layers)
    arr = (RcwaCell * n)(*layers)
    N = (2 * layers[0].Mx + 1) * (2 * layers[0].My + 1)
    ex = np.array([complex(Ex0).real, complex(Ex0).imag])
    ey = np.array([complex(Ey0).real, complex(Ey0).imag])
    out = RcwaResult()
    orders = (RcwaOrder * N)()
    check(load().celeris_solve_rcwa_2d_orders(arr, n, _dp(ex), _dp(ey), ctypes.byref(out), orders, N))
    return result_dict(out), [dict(p=o.p, q=o.q, de_t=o.de_t, de_r=o.de_r, prop_t=bool(o.prop_t),
                                   prop_r=bool(o.prop_r)) for o in orders]


def eig_general(A):
    """Eigenpairs of one complex matrix or a stack [count, n, n]: (evals, evecs, info),
    evecs[..., :, i] the unit-norm eigenvector of evals[..., i]."""
    A = np.asarray(A, dtype=np.complex128)
    single = A.ndim == 2
    A3 = A[None] if single else A
    count, n = A3.shape[0], A3.shape[1]
    colmajor = np.ascontiguousarray(np.transpose(A3, (0, 2, 1)))  # Fortran order per matrix
    vals = np.zeros((count, n), dtype=np.complex128)
    vecs = np.zeros((count, n, n), dtype=np.complex128)  # column-major per matrix: [count, col, row]
    info = np.zeros(count, dtype=np.int32)
    check(load().celeris_eig_general_batch(_dp(colmajor.view(np.float64)), n, count, _dp(vals.view(np.float64)),
                                           _dp(vecs.view(np.float64)), info.ctypes.data_as(_PI)))
    vecs = np.transpose(vecs, (0, 2, 1))
    return (vals[0], vecs[0], info[0]) if single else (vals, vecs, info)
