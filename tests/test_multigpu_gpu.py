"""The multi-device forms of celeris_b200.multigpu through the kernels, on the
GPUs this run has. With one GPU, "devices" [0, 0] runs two row blocks (or two
cell shards) from two host threads on the same device: independent launches
that never wait on each other. The split results must equal the one-call
results (far field and adjoint to the FP64 rounding of the chunk sums, RCWA
exactly)."""
import numpy as np
import pytest

from celeris_b200 import capi
from celeris_b200 import multigpu as MG
from celeris_b200.workloads import metalens_70k, rcwa_uneven_4096

pytestmark = pytest.mark.gpu


def _devices():
    import torch

    n = torch.cuda.device_count()
    return list(range(n)) if n > 1 else [0, 0]


@pytest.mark.parametrize("form", [capi.FORM_PLAIN_F64, capi.FORM_F32C], ids=["plain_f64", "f32c"])
def test_field_and_adjoint_split_over_devices(form):
    import torch

    from celeris_b200 import torch_ops as T

    ap, g = metalens_70k()
    grid = T.FarFieldGrid(g.n, g.half_window_um, g.z_um, ap.wavelength_um)
    dev = torch.device("cuda", 0)
    px, py, t = (torch.tensor(v, device=dev) for v in (ap.px, ap.py, ap.t))
    whole = T.rs_field_dev(px, py, t, grid, form)
    split = MG.rs_field_multi(ap.px, ap.py, ap.t, grid, form, devices=_devices())
    w = whole.cpu().numpy()
    assert np.max(np.abs(split.cpu().numpy() - w)) <= 1e-12 * np.max(np.abs(w))
    v = torch.conj(whole) / whole.abs().max()
    adj = T.rs_adjoint_dev(px, py, v, grid, form).cpu().numpy()
    adj_split = MG.rs_adjoint_multi(ap.px, ap.py, v, grid, form, devices=_devices()).cpu().numpy()
    # the adjoint tiles the pixels, so a row split regroups its FP32 tile sums in
    # the precision form: there the split agrees to that form's accuracy
    # against the FP64 adjoint (1e-5 of the largest output), in FP64 to rounding
    if form == capi.FORM_F32C:
        adj64 = T.rs_adjoint_dev(px, py, v, grid, capi.FORM_PLAIN_F64).cpu().numpy()
        assert np.max(np.abs(adj_split - adj64)) <= 1e-5 * np.max(np.abs(adj64))
    else:
        assert np.max(np.abs(adj_split - adj)) <= 1e-12 * np.max(np.abs(adj))


def test_rcwa_batch_split_over_devices():
    cells = [capi.rcwa_cell(**c) for c in rcwa_uneven_4096()[:48]]
    ref, info = capi.rcwa_batch(cells)
    got, info2 = MG.rcwa_batch_multi(cells, devices=_devices())
    assert np.all(info == 0) and np.all(info2 == 0)
    for a, b in zip(got, ref):
        assert abs(a["tx0"] - b["tx0"]) <= 1e-12 * abs(b["tx0"])
        assert abs(a["R"] - b["R"]) <= 1e-12
