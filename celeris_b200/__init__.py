"""celeris_b200 - B200-native hot path of the CELERIS metalens engine.

The far-field Rayleigh-Sommerfeld sum and the 2D RCWA unit-cell solves run as
hand-written sm_100a kernels behind the C ABI in include/celeris_b200.h
(libceleris_b200.so). This package exposes:

  * ``capi``       - the C ABI through ctypes (the boundary a caller binds);
  * the reference's Python surface (``solve_rcwa_2d``, ``build_unit_cell_library``,
    ``compute_psf``, ``analyze_focus``, ``Material``, ...) from the C++ host
    mirror ``_celeris``;
  * ``torch_ops``  - the far-field as a torch.autograd.Function (adjoint kernel);
  * ``multigpu``   - one focal grid, one adjoint or one RCWA batch split over
    several devices;
  * ``workloads``  - seeded synthetic inputs with the shapes of the measured
    workloads.

Importing the package loads no native library: ``capi`` loads
libceleris_b200.so at its first call, and the reference-API names load the host
mirror ``_celeris`` (which links libceleris_b200.so) at their first use. So a
process that only needs ``workloads`` maps none of the product's libraries.
Nothing here falls back to CPU arithmetic: a missing or unloadable library is an
error at first use.
"""
from __future__ import annotations

import importlib

__version__ = "0.1.0"

_SUBMODULES = ("capi", "torch_ops", "workloads", "multigpu")


def _host_mirror():
    return importlib.import_module("._celeris", __name__)


def __getattr__(name):
    if name in _SUBMODULES:
        return importlib.import_module("." + name, __name__)
    if name == "_celeris":
        return _host_mirror()
    if name.startswith("__"):
        raise AttributeError(name)
    try:
        value = getattr(_host_mirror(), name)
    except AttributeError:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}") from None
    globals()[name] = value
    return value


def __dir__():
    names = set(globals()) | set(_SUBMODULES)
    try:
        names |= {n for n in dir(_host_mirror()) if not n.startswith("_")}
    except ImportError:
        pass
    return sorted(names)
