"""The far-field sum as differentiable torch operations.

RSField: t (complex128 [npil], CUDA) -> E (complex128 [n, n]) through
celeris_rs_field_dev; its backward is the hand-written adjoint kernel
celeris_rs_adjoint_dev (conjugate-transpose pixel -> pillar sum, pixel tiles
recomputed, never stored), which is exactly PyTorch's vector-Jacobian product
for a C-linear map: grad_t = G^H grad_E.

LibrarySpline: per-pillar fill w -> complex t(w) = A(w) exp(i phi(w)) by natural
cubic splines of amplitude and unwrapped phase over a unit-cell library (the
fill -> (t, phi) chain of the inverse-design gradient). The reference has no
far-field gradient; its only gradient is central finite differences of RCWA
(src/celeris/design/optimize.cpp:60-71).

All device work goes through libceleris_b200.so; the torch tensors are device
memory and streams only.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import capi


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class FarFieldGrid:
    """Focal grid of n x n pixels over [c - W, c + W]^2 at distance z."""

    def __init__(self, n: int, half_window_um: float, z_um: float, wavelength_um: float,
                 cx: float = 0.0, cy: float = 0.0):
        self.n = int(n)
        self.W = float(half_window_um)
        self.z = float(z_um)
        self.wavelength = float(wavelength_um)
        self.k = 2.0 * np.pi / self.wavelength
        self.cx = float(cx)
        self.cy = float(cy)

    def coords(self, device=None):
        step = 2.0 * self.W / (self.n - 1)
        i = torch.arange(self.n, dtype=torch.float64, device=device)
        fx = self.cx - self.W + i * step
        fy = self.cy - self.W + i * step
        return fx, fy


def rs_field_dev(px, py, t, grid: FarFieldGrid, form=capi.FORM_PLAIN_F64, want_intensity=False):
    """Forward far-field on device tensors (no autograd). Returns E (and |E|^2)."""
    lib = capi.load()
    E = torch.empty((grid.n, grid.n), dtype=torch.complex128, device=t.device)
    inten = torch.empty((grid.n, grid.n), dtype=torch.float64, device=t.device) if want_intensity else None
    capi.check(lib.celeris_rs_field_dev(form, _ptr(px), _ptr(py), _ptr(t), int(px.numel()), grid.cx, grid.cy,
                                        grid.z, grid.k, grid.n, grid.W, _ptr(E),
                                        _ptr(inten) if inten is not None else None, _stream()))
    return (E, inten) if want_intensity else E


def rs_adjoint_dev(px, py, v, grid: FarFieldGrid, form=capi.FORM_PLAIN_F64):
    """out_j = sum_p conj(g_pj) v_p in the plain FP64 or the precision (packed FP32,
    compensated sums, e^{-ikz} in FP64) form."""
    lib = capi.load()
    out = torch.empty(px.numel(), dtype=torch.complex128, device=v.device)
    v = v.contiguous()
    capi.check(lib.celeris_rs_adjoint_dev(form, _ptr(px), _ptr(py), int(px.numel()), grid.cx,
                                          grid.cy, grid.z, grid.k, grid.n, grid.W, _ptr(v), _ptr(out),
                                          _stream()))
    return out


class RSField(torch.autograd.Function):
    @staticmethod
    def forward(ctx, t, px, py, grid, form):
        t = t.contiguous()
        ctx.save_for_backward(px, py)
        ctx.grid = grid
        ctx.form = form
        return rs_field_dev(px, py, t, grid, form)

    @staticmethod
    def backward(ctx, grad_E):
        # the adjoint runs in the forward's form
        px, py = ctx.saved_tensors
        g = grad_E.to(torch.complex128).contiguous()
        return rs_adjoint_dev(px, py, g, ctx.grid, ctx.form), None, None, None, None


def rs_field(t, px, py, grid: FarFieldGrid, form=capi.FORM_PLAIN_F64):
    """Differentiable far-field: E = G t on `grid` (complex128 CUDA tensors)."""
    for a in (t, px, py):
        if not a.is_cuda:
            raise capi.CelerisError(capi.ERR_INVALID_ARG, "rs_field expects CUDA tensors")
    return RSField.apply(t, px.contiguous(), py.contiguous(), grid, form)


# ---- fill -> complex transmission (natural cubic spline) ---------------------
def natural_spline_coeffs(x: np.ndarray, y: np.ndarray):
    """Coefficients (a, b, c, d) per interval for a natural cubic spline through
    (x, y): s(u) = a + b h + c h^2 + d h^3 with h = u - x_i."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    m = len(x)
    h = np.diff(x)
    A = np.zeros((m, m))
    rhs = np.zeros(m)
    A[0, 0] = A[-1, -1] = 1.0
    for i in range(1, m - 1):
        A[i, i - 1] = h[i - 1]
        A[i, i] = 2.0 * (h[i - 1] + h[i])
        A[i, i + 1] = h[i]
        rhs[i] = 3.0 * ((y[i + 1] - y[i]) / h[i] - (y[i] - y[i - 1]) / h[i - 1])
    c = np.linalg.solve(A, rhs)
    b = (y[1:] - y[:-1]) / h - h * (2.0 * c[:-1] + c[1:]) / 3.0
    d = (c[1:] - c[:-1]) / (3.0 * h)
    return np.stack([y[:-1], b, c[:-1], d], axis=1)  # [m-1, 4]


class LibrarySpline:
    """Complex t(w) from a library (fill, amplitude, phase) by natural cubic
    splines of amplitude and unwrapped phase. Evaluated with torch ops so the
    chain rule to the fills is automatic."""

    def __init__(self, fill, amplitude, phase, device="cuda"):
        fill = np.asarray(fill, np.float64)
        self.fill = fill
        self.amp_c = torch.tensor(natural_spline_coeffs(fill, amplitude), device=device)
        self.ph_c = torch.tensor(natural_spline_coeffs(fill, np.unwrap(np.asarray(phase, np.float64))), device=device)
        self.knots = torch.tensor(fill, device=device)

    def _eval(self, coef, w):
        i = torch.clamp(torch.searchsorted(self.knots, w.detach(), right=True) - 1, 0, coef.shape[0] - 1)
        h = w - self.knots[i]
        c = coef[i]
        return c[:, 0] + h * (c[:, 1] + h * (c[:, 2] + h * c[:, 3]))

    def __call__(self, w):
        amp = self._eval(self.amp_c, w)
        ph = self._eval(self.ph_c, w)
        return torch.polar(amp, ph)

    def numpy_eval(self, w):
        """The same spline on the host in float64 (for finite-difference checks)."""
        w = np.asarray(w, np.float64)
        kn = self.fill
        i = np.clip(np.searchsorted(kn, w, side="right") - 1, 0, len(kn) - 2)
        h = w - kn[i]

        def ev(c):
            c = c.cpu().numpy()[i]
            return c[:, 0] + h * (c[:, 1] + h * (c[:, 2] + h * c[:, 3]))

        return ev(self.amp_c) * np.exp(1j * ev(self.ph_c))


def encircled_energy_loss(E: torch.Tensor, grid: FarFieldGrid, radius_um: float = 1.0):
    """L = -(sum of |E|^2 within radius of the axis) / (sum of |E|^2)."""
    fx, fy = grid.coords(E.device)
    r2 = fy[:, None] ** 2 + fx[None, :] ** 2
    mask = (r2 <= radius_um * radius_um).to(torch.float64)
    inten = E.real ** 2 + E.imag ** 2
    return -(inten * mask).sum() / inten.sum()
