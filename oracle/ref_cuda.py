"""ORACLE - test infrastructure only (bench.py's GPU comparator leg).

ctypes access to oracle/_ref/libref_psf_cuda.so: the REFERENCE's own FP32 CUDA
far-field kernel psf_kernel and its wrapper propagate_psf
(src/celeris/cuda/propagate.cu:36-84, 133-193), compiled unmodified for sm_100a
by oracle/Makefile. The product never loads this library.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_psf_cuda.so")
_P = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_V = ctypes.c_void_p
_D = ctypes.c_double
_lib = None


def available() -> bool:
    return os.path.exists(_PATH)


def load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(_PATH)
        _lib.ref_cuda_propagate_psf.argtypes = [_P, _P, _P, ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _D, _P]
        _lib.ref_cuda_propagate_psf.restype = ctypes.c_int
        _lib.ref_cuda_psf_kernel.argtypes = [_V, _V, _V, _V, ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _D, _V,
                                             ctypes.c_int, _F]
        _lib.ref_cuda_psf_kernel.restype = ctypes.c_int
    return _lib


def propagate_psf(px, py, t, cx, cy, z, k, n, half_window):
    """The reference's public GPU call: |E|^2 (n x n, float64) from host buffers."""
    px = np.ascontiguousarray(px, dtype=np.float64)
    py = np.ascontiguousarray(py, dtype=np.float64)
    t = np.ascontiguousarray(t, dtype=np.complex128)
    out = np.empty((n, n), dtype=np.float64)
    st = load().ref_cuda_propagate_psf(px.ctypes.data_as(_P), py.ctypes.data_as(_P),
                                       t.view(np.float64).ctypes.data_as(_P), len(px), cx, cy, z, k, n,
                                       half_window, out.ctypes.data_as(_P))
    if st != 0:
        raise RuntimeError("reference propagate_psf returned false")
    return out


def psf_kernel(px, py, t, cx, cy, z, k, n, half_window, reps=1):
    """The reference kernel alone on device buffers (torch float32 tensors on the
    current device), `reps` timed launches. Returns (|E|^2 as float64 numpy,
    ms per launch)."""
    import torch

    dev = torch.device("cuda")
    x = torch.tensor(np.asarray(px, dtype=np.float32), device=dev)
    y = torch.tensor(np.asarray(py, dtype=np.float32), device=dev)
    tr = torch.tensor(np.asarray(np.real(t), dtype=np.float32), device=dev)
    ti = torch.tensor(np.asarray(np.imag(t), dtype=np.float32), device=dev)
    out = torch.empty((n, n), dtype=torch.float32, device=dev)
    ms = ctypes.c_float(0.0)
    torch.cuda.synchronize()
    st = load().ref_cuda_psf_kernel(x.data_ptr(), y.data_ptr(), tr.data_ptr(), ti.data_ptr(), len(px), cx, cy, z, k,
                                    n, half_window, out.data_ptr(), reps, ctypes.byref(ms))
    if st != 0:
        raise RuntimeError(f"reference psf_kernel launch failed ({st})")
    return out.double().cpu().numpy(), float(ms.value)
