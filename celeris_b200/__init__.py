"""celeris_b200 - B200-native hot path of the CELERIS metalens engine.

The far-field Rayleigh-Sommerfeld sum and the 2D RCWA unit-cell solves run as
hand-written sm_100a kernels behind the C ABI in include/celeris_b200.h
(libceleris_b200.so). This package exposes:

  * ``capi``       - the C ABI through ctypes (the boundary a caller binds);
  * the reference's Python surface (``solve_rcwa_2d``, ``build_unit_cell_library``,
    ``compute_psf``, ``analyze_focus``, ``Material``, ...) from the C++ host
    mirror ``_celeris`` when it is built;
  * ``torch_ops``  - the far-field as a torch.autograd.Function (adjoint kernel).

Nothing here falls back to CPU arithmetic: a missing or unloadable library is an
error.
"""
from __future__ import annotations

__version__ = "0.1.0"

from . import capi  # noqa: F401  (ctypes boundary; the library loads on first use)

try:  # the C++ host mirror of the reference API (pybind11)
    from ._celeris import *  # noqa: F401,F403
    from . import _celeris  # noqa: F401
except ImportError as _e:  # pragma: no cover - only before build()
    _celeris = None
    _celeris_import_error = _e
