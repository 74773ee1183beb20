"""Inverse design: the adjoint far-field kernel behind torch.autograd.

Loss L = -(|E|^2 within 1 um of the axis) / (sum of |E|^2) on the 161^2 grid
of the 70,688-pillar metalens; per-pillar fills w -> t(w) by natural cubic
splines over the 64-width library (solved on the GPU). The float64 gradient
dL/dw from the adjoint kernel is checked against central finite differences
(h = 1e-6) of the oracle loss on 32 random pillars (<= 1e-6 relative), and
against the reference's own gradient method (central differences of
solve_rcwa_2d, optimize.cpp:52-71) for dt/dfill at library nodes.
"""
import math

import numpy as np
import pytest

from celeris_b200 import capi
from celeris_b200.workloads import metalens_70k, rcwa_library_64
from oracle import farfield as F

pytestmark = pytest.mark.gpu


def library():
    cells = rcwa_library_64()
    res, info = capi.rcwa_batch([capi.rcwa_cell(**c) for c in cells])
    assert np.all(info == 0)
    fill = np.array([c["fill_x"] for c in cells])
    t = np.array([res[2 * i]["tx0"] for i in range(len(cells))])
    return fill, np.abs(t), np.angle(t)


def setup():
    import torch

    from celeris_b200 import torch_ops as T

    ap, g = metalens_70k()
    fill, amp, ph = library()
    spline = T.LibrarySpline(fill, amp, ph)
    grid = T.FarFieldGrid(g.n, g.half_window_um, g.z_um, ap.wavelength_um)
    rng = np.random.default_rng(0)
    w0 = rng.uniform(fill[1], fill[-2], ap.npil)
    dev = torch.device("cuda")
    px = torch.tensor(ap.px, device=dev)
    py = torch.tensor(ap.py, device=dev)
    return ap, g, spline, grid, w0, px, py


def loss_and_grad(spline, grid, w0, px, py):
    import torch

    from celeris_b200 import torch_ops as T

    w = torch.tensor(w0, device="cuda", requires_grad=True)
    E = T.rs_field(spline(w), px, py, grid)
    L = T.encircled_energy_loss(E, grid, 1.0)
    L.backward()
    return float(L.detach()), w.grad.cpu().numpy(), E.detach().cpu().numpy()


def fd_oracle(ap, g, spline, w0, idx, h=1e-6):
    """Central differences of the oracle loss, evaluated without cancellation:
    the field is linear in t, so E(w_j +/- h) = E + g_j dT and the change of
    the masked and total energies is formed directly."""
    t0 = spline.numpy_eval(w0)
    k = 2 * math.pi / ap.wavelength_um
    E = F.rs_field(ap.px, ap.py, t0, 0.0, 0.0, g.z_um, k, g.n, g.half_window_um)
    step = 2 * g.half_window_um / (g.n - 1)
    c = -g.half_window_um + np.arange(g.n) * step
    fy, fx = np.meshgrid(c, c, indexing="ij")
    mask = (fx * fx + fy * fy) <= 1.0
    I = np.abs(E) ** 2
    In, Tot = I[mask].sum(), I.sum()
    out = []
    for j in idx:
        R = np.sqrt((fx - ap.px[j]) ** 2 + (fy - ap.py[j]) ** 2 + g.z_um ** 2)
        gj = np.exp(1j * k * R) / R
        dl = []
        for s in (+1, -1):
            dT = spline.numpy_eval(np.array([w0[j] + s * h]))[0] - t0[j]
            d = gj * dT
            dI = 2 * np.real(np.conj(E) * d) + np.abs(d) ** 2
            dIn, dTot = dI[mask].sum(), dI.sum()
            dl.append((In * dTot - Tot * dIn) / (Tot * (Tot + dTot)))
        out.append((dl[0] - dl[1]) / (2 * h))
    return np.array(out), -In / Tot


def test_adjoint_gradient_matches_central_differences():
    ap, g, spline, grid, w0, px, py = setup()
    L, grad, _ = loss_and_grad(spline, grid, w0, px, py)
    idx = np.random.default_rng(1).choice(ap.npil, 32, replace=False)
    fd, L_oracle = fd_oracle(ap, g, spline, w0, idx)
    assert abs(L - L_oracle) <= 1e-12 * abs(L_oracle)
    rel = np.max(np.abs(grad[idx] - fd)) / np.max(np.abs(fd))
    assert rel <= 1e-6, rel
    big = np.abs(fd) > 1e-2 * np.max(np.abs(fd))
    assert np.all(np.abs(grad[idx][big] - fd[big]) <= 1e-6 * np.abs(fd[big]))


def test_library_derivative_vs_reference_style_fd():
    """dt/dfill of the spline against the reference's gradient method: central
    differences of the RCWA solve in fill (h = 5e-3 as optimize.cpp:52, and
    1e-4). Loose: it measures interpolation error, not arithmetic."""
    import torch

    fill, amp, ph = library()
    from celeris_b200 import torch_ops as T

    spline = T.LibrarySpline(fill, amp, ph)
    base = rcwa_library_64()[0]
    for i in (10, 30, 50):
        w = torch.tensor([fill[i]], device="cuda", requires_grad=True)
        t = spline(w)
        (gr,) = torch.autograd.grad(t.real.sum(), w, retain_graph=True)
        (gi,) = torch.autograd.grad(t.imag.sum(), w)
        dt_spline = complex(float(gr), float(gi))
        for h, tol in ((5e-3, 1e-2), (1e-4, 2e-3)):
            cells = [dict(base, fill_x=fill[i] + h), dict(base, fill_x=fill[i] - h)]
            res, _ = capi.rcwa_batch([capi.rcwa_cell(**c) for c in cells])
            dt_fd = (res[0]["tx0"] - res[2]["tx0"]) / (2 * h)
            assert abs(dt_spline - dt_fd) <= tol * abs(dt_fd), (i, h, dt_spline, dt_fd)


def test_adam_200_steps_improves_encircled_energy():
    import torch

    from celeris_b200 import torch_ops as T

    ap, g, spline, grid, w0, px, py = setup()
    w = torch.tensor(w0, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([w], lr=1e-3)
    first = None
    for _ in range(200):
        opt.zero_grad()
        L = T.encircled_energy_loss(T.rs_field(spline(w), px, py, grid), grid, 1.0)
        L.backward()
        opt.step()
        with torch.no_grad():
            w.clamp_(float(spline.fill[0]), float(spline.fill[-1]))
        if first is None:
            first = float(L)
    assert float(L) < first
