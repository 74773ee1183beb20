"""Per-thread resources of the host-buffer entry points are released when the
calling thread exits. Each calling thread gets its own CUDA streams, events,
device workspace arenas, device I/O buffer and pinned staging (the reference
calls its solvers from short-lived std::async workers, metalens.cpp:153-161).

Calls made from a series of short-lived threads must return what the same
calls return on the main thread, and must leave device memory where the
previous thread left it."""
import threading

import numpy as np
import pytest

from celeris_b200 import capi
from celeris_b200.workloads import metalens_70k

pytestmark = pytest.mark.gpu

COMMON = dict(period_um=0.4, wavelength_um=0.633, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0)


def _device_free():
    import torch  # free bytes on the device, the library's own cudaMalloc arenas included

    return torch.cuda.mem_get_info(0)[0]


def _calls():
    """One call of each host-buffer path: far field (precision form, stated
    error on a second stream), an RCWA batch, a two-layer stack, eigensolves."""
    ap, g = metalens_70k()
    E, _, err = capi.rs_field(ap.px, ap.py, ap.t, 0.0, 0.0, g.z_um, ap.k, g.n, g.half_window_um,
                              form=capi.FORM_F32C, want_intensity=False, want_err=True)
    cells = [capi.rcwa_cell(**COMMON, fill_x=0.2 + 0.01 * i, thickness_um=0.6, Mx=5) for i in range(48)]
    res, info = capi.rcwa_batch(cells)
    stack = [capi.rcwa_cell(**COMMON, fill_x=0.5, thickness_um=0.3, Mx=3),
             capi.rcwa_cell(**COMMON, fill_x=0.35, thickness_um=0.2, Mx=3)]
    sres, sinfo = capi.rcwa_stack_batch([stack])
    A = np.random.default_rng(3).standard_normal((8, 60, 60)) + 0j
    vals, _, einfo = capi.eig_general(A)
    assert not np.any(info) and not np.any(sinfo) and not np.any(einfo)
    return dict(E=E, err=err, tx=np.array([r["tx0"] for r in res]), stx=np.array([r["tx0"] for r in sres]),
                vals=np.sort_complex(np.asarray(vals).ravel()))


def test_results_and_device_memory_across_short_lived_threads():
    ref = _calls()
    free = []
    for i in range(6):
        out = []
        th = threading.Thread(target=lambda: out.append(_calls()))
        th.start()
        th.join()
        assert len(out) == 1
        for key in ref:
            assert np.array_equal(out[0][key], ref[key]), key
        free.append(_device_free())
    # Each thread allocates its own arenas (the 48-cell batch alone ~360 MB);
    # none may outlive the thread, so after two warm-up threads (one-time
    # context allocations of the process) free memory stays put.
    steady = free[2:]
    assert max(steady) - min(steady) < (32 << 20), [f >> 20 for f in free]
