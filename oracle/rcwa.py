"""ORACLE - test infrastructure only (the checker and the CPU port timed as the
RCWA cpu_baseline). The product path never imports this module.

numpy/scipy restatement of the reference's 2D vectorial RCWA,
src/celeris/rcwa/rcwa2d.cpp:14-488, following its steps in order:
  orders and wavevectors            rcwa2d.cpp:103-105, 224-252
  homogeneous regions               rcwa2d.cpp:255-271 (grazing guard 260, branch 126)
  patterned region, plain rect      rcwa2d.cpp:280-333 (Li inverse rule, analytic Fourier)
  patterned region, other shapes    rcwa2d.cpp:74-95 (4x4 supersampled raster), 147-205
                                    (separable centred DFT, Laurent Toeplitz, inverse),
                                    337 (grid = max(128, 8(2M+1)))
  kp, ep2, eigenproblem             rcwa2d.cpp:346-365 (M = ep2 kp - kkT, q = branch(sqrt))
  S-matrix recursion                rcwa2d.cpp:376-401 (grcwa GetSMatrix)
  excitation, flux, efield, output  rcwa2d.cpp:403-463
The dense eigensolve is scipy.linalg.eig (LAPACK zgeev), i.e. the reference's
CELERIS_USE_LAPACK build (src/celeris/rcwa/eig.cpp:52-78); the reference's
default Eigen ComplexEigenSolver (eig.cpp:87-92) is a third-party dependency
(Eigen 3.4.0, CMakeLists.txt:56-71) absent here. The results are invariant to
eigenvector scaling and ordering (eig.hpp:16-18).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla

PI = math.pi

RECT, ELLIPSE, CROSS, RING = 0, 1, 2, 3


def order_index(p, q, Mx, My):
    return (p + Mx) * (2 * My + 1) + (q + My)


def rect1d(m, fill):
    m = np.asarray(m)
    out = np.where(m == 0, fill, np.sin(PI * m * fill) / (PI * np.where(m == 0, 1, m)))
    return out


def branch(q):
    """grcwa branch: keep Im(kz) >= 0 (rcwa2d.cpp:126)."""
    q = np.asarray(q, dtype=np.complex128)
    return np.where(q.imag < 0.0, -q, q)


def inside(xf, yf, shape, fill_x, fill_y, shape_param, rotation):
    """RectCell2D::inside (rcwa2d.cpp:37-72), vectorised over sample points."""
    if rotation != 0.0:
        c, s = math.cos(rotation), math.sin(rotation)
        xr = c * xf + s * yf
        yr = -s * xf + c * yf
        xf, yf = xr, yr
    ax, ay = fill_x * 0.5, fill_y * 0.5
    if shape == RECT:
        return (np.abs(xf) <= ax) & (np.abs(yf) <= ay)
    if shape == ELLIPSE:
        if ax <= 0 or ay <= 0:
            return np.zeros_like(xf, dtype=bool)
        u, v = xf / ax, yf / ay
        return u * u + v * v <= 1.0
    if shape == CROSS:
        hx, hy = ax * shape_param, ay * shape_param
        vbar = (np.abs(xf) <= hx) & (np.abs(yf) <= ay)
        hbar = (np.abs(yf) <= hy) & (np.abs(xf) <= ax)
        return vbar | hbar
    if shape == RING:
        if ax <= 0 or ay <= 0:
            return np.zeros_like(xf, dtype=bool)
        u, v = xf / ax, yf / ay
        r2 = u * u + v * v
        ri = shape_param
        return (r2 <= 1.0) & (r2 >= ri * ri)
    raise ValueError(shape)


def rasterize_eps(eps_p, eps_b, ngx, ngy, shape, fill_x, fill_y, shape_param, rotation):
    """RectCell2D::rasterize_eps (rcwa2d.cpp:74-95): 4x4 supersampled inside
    fraction per pixel, eps = eb + (ep - eb) * frac, row-major [iy, ix]."""
    S = 4
    ix = np.arange(ngx)[None, :, None, None]
    iy = np.arange(ngy)[:, None, None, None]
    sx = np.arange(S)[None, None, None, :]
    sy = np.arange(S)[None, None, :, None]
    xf = (ix + (sx + 0.5) / S) / ngx - 0.5
    yf = (iy + (sy + 0.5) / S) / ngy - 0.5
    xf, yf = np.broadcast_arrays(xf, yf)
    hit = inside(xf, yf, shape, fill_x, fill_y, shape_param, rotation).sum(axis=(2, 3))
    frac = hit / float(S * S)
    return eps_b + (eps_p - eps_b) * frac


def laurent_toeplitz(eps, ngx, ngy, Mx, My):
    """shape_operators' epsT (rcwa2d.cpp:147-198): centred separable DFT of the
    sampled eps up to +/-2M, gathered into the Laurent Toeplitz matrix."""
    def phase_table(ng, mmax):
        m = np.arange(-mmax, mmax + 1)[:, None]
        xf = (np.arange(ng) + 0.5) / ng - 0.5
        return np.exp(-2j * PI * m * xf[None, :]) / ng  # [2mmax+1, ng]

    PX = phase_table(ngx, 2 * Mx)
    PY = phase_table(ngy, 2 * My)
    G1 = eps @ PX.T            # [ngy, 4Mx+1]  (sum over ix)
    Ge = (PY @ G1).T           # [4Mx+1, 4My+1]  Ge[dp, dq]
    nx, ny = 2 * Mx + 1, 2 * My + 1
    p = np.repeat(np.arange(-Mx, Mx + 1), ny)
    q = np.tile(np.arange(-My, My + 1), nx)
    dp = p[:, None] - p[None, :]
    dq = q[:, None] - q[None, :]
    return Ge[dp + 2 * Mx, dq + 2 * My]


def rect_operators(eps_p, eps_b, fx, fy, Mx, My):
    """Einv, Exx, Eyy of the analytic Li path (rcwa2d.cpp:280-333)."""
    nx, ny = 2 * Mx + 1, 2 * My + 1
    ipe, ibe = 1.0 / eps_p, 1.0 / eps_b
    p = np.repeat(np.arange(-Mx, Mx + 1), ny)
    q = np.tile(np.arange(-My, My + 1), nx)
    dp = p[:, None] - p[None, :]
    dq = q[:, None] - q[None, :]
    Sx = rect1d(dp, fx)
    Sy = rect1d(dq, fy)
    Einv = (ipe - ibe) * (Sx * Sy)
    Einv = Einv + np.where((dp == 0) & (dq == 0), ibe, 0.0)
    a = np.arange(-Mx, Mx + 1)
    Hx = np.where(a[:, None] == a[None, :], ibe, 0.0) + (ipe - ibe) * rect1d(a[:, None] - a[None, :], fx)
    Axb = np.linalg.inv(Hx)
    b = np.arange(-My, My + 1)
    Hy = np.where(b[:, None] == b[None, :], ibe, 0.0) + (ipe - ibe) * rect1d(b[:, None] - b[None, :], fy)
    Ayb = np.linalg.inv(Hy)
    sy = rect1d(dq, fy)
    Exx = Axb[p[:, None] + Mx, p[None, :] + Mx] * sy
    Exx = Exx + np.where(dp == 0, eps_b * (np.where(dq == 0, 1.0, 0.0) - sy), 0.0)
    sx = rect1d(dp, fx)
    Eyy = Ayb[q[:, None] + My, q[None, :] + My] * sx
    Eyy = Eyy + np.where(dq == 0, eps_b * (np.where(dp == 0, 1.0, 0.0) - sx), 0.0)
    return Einv.astype(np.complex128), Exx.astype(np.complex128), Eyy.astype(np.complex128)


def solve(n_inc, layers, n_sub, period_x, period_y, wavelength, theta, phi, Ex0, Ey0, Mx, My,
          orders_out=False, eig=None):
    """solve_rcwa_2d (rcwa2d.cpp:209-488). `layers`: dicts with eps_pillar, eps_bg,
    fill_x, fill_y, thickness, shape, shape_param, rotation, and optional grid
    (raster size override) / force_laurent. Returns a dict like Rcwa2DResult."""
    if Mx < 0 or My < 0:
        raise ValueError("M must be >= 0")
    if not layers:
        raise ValueError("solve_rcwa_2d: stack has no layers")
    eig = eig or (lambda A: sla.eig(A, left=False, right=True, check_finite=False))
    N = (2 * Mx + 1) * (2 * My + 1)
    k0 = 2.0 * PI / wavelength
    omega = complex(k0)
    omega2 = omega * omega
    n_inc = complex(n_inc)
    n_sub = complex(n_sub)
    kx0 = n_inc * math.sin(theta) * math.cos(phi) * omega
    ky0 = n_inc * math.sin(theta) * math.sin(phi) * omega
    p = np.repeat(np.arange(-Mx, Mx + 1), 2 * My + 1)
    q = np.tile(np.arange(-My, My + 1), 2 * Mx + 1)
    kxv = kx0 - 2.0 * PI * p / period_x
    kyv = ky0 - 2.0 * PI * q / period_y
    Kx = np.diag(kxv.astype(np.complex128))
    Ky = np.diag(kyv.astype(np.complex128))
    Id = np.eye(N, dtype=np.complex128)
    kkT = np.block([[Kx @ Kx, Kx @ Ky], [Ky @ Kx, Ky @ Ky]])

    def uniform_region(nreg, thick):
        er = nreg * nreg
        ier = 1.0 / er
        kz = np.sqrt(er * omega2 - kxv * kxv - kyv * kyv + 0j)
        kz = np.where(np.abs(kz) < 1e-8, 1e-8j, kz)
        kz = branch(kz)
        qv = np.concatenate([kz, kz])
        kp = np.block([[omega2 * Id - ier * (Ky @ Ky), ier * (Ky @ Kx)],
                       [ier * (Kx @ Ky), omega2 * Id - ier * (Kx @ Kx)]])
        return dict(q=qv, phi=np.eye(2 * N, dtype=np.complex128), kp=kp, thickness=thick)

    def patterned_region(L):
        ep, eb = complex(L["eps_pillar"]), complex(L["eps_bg"])
        shape = L.get("shape", RECT)
        rot = L.get("rotation", 0.0)
        plain_rect = shape == RECT and rot == 0.0 and not L.get("force_laurent", False)
        if plain_rect:
            Einv, Exx, Eyy = rect_operators(ep, eb, L["fill_x"], L["fill_y"], Mx, My)
        else:
            ng = L.get("grid") or max(128, 8 * (2 * max(Mx, My) + 1))
            eps = rasterize_eps(ep, eb, ng, ng, shape, L["fill_x"], L["fill_y"], L.get("shape_param", 0.5), rot)
            epsT = laurent_toeplitz(eps, ng, ng, Mx, My)
            Exx = epsT
            Eyy = epsT
            Einv = np.linalg.inv(epsT)
        kp = np.block([[omega2 * Id - Ky @ Einv @ Ky, Ky @ Einv @ Kx],
                       [Kx @ Einv @ Ky, omega2 * Id - Kx @ Einv @ Kx]])
        ep2 = np.zeros((2 * N, 2 * N), dtype=np.complex128)
        ep2[:N, :N] = Eyy
        ep2[N:, N:] = Exx
        evals, phiv = eig(ep2 @ kp - kkT)
        qv = branch(np.sqrt(evals.astype(np.complex128)))
        return dict(q=qv, phi=phiv, kp=kp, thickness=L["thickness"])

    R = [uniform_region(n_inc, 0.0)] + [patterned_region(L) for L in layers] + [uniform_region(n_sub, 0.0)]
    NL = len(R)
    N2 = 2 * N
    S11 = np.eye(N2, dtype=np.complex128)
    S12 = np.zeros((N2, N2), dtype=np.complex128)
    S21 = np.zeros((N2, N2), dtype=np.complex128)
    S22 = np.eye(N2, dtype=np.complex128)
    for li in range(NL - 1):
        a, b = R[li], R[li + 1]
        Q = np.linalg.inv(a["phi"]) @ b["phi"]
        P1 = np.diag(a["q"]) @ np.linalg.inv(a["kp"] @ a["phi"])
        P2 = (b["kp"] @ b["phi"]) @ np.diag(1.0 / b["q"])
        P = P1 @ P2
        T11 = 0.5 * (Q + P)
        T12 = 0.5 * (Q - P)
        d1 = np.diag(np.exp(1j * a["q"] * a["thickness"]))
        d2 = np.diag(np.exp(1j * b["q"] * b["thickness"]))
        Pinv = np.linalg.inv(T11 - d1 @ S12 @ T12)
        nS11 = Pinv @ d1 @ S11
        nS12 = Pinv @ (d1 @ S12 @ T11 - T12) @ d2
        nS21 = S21 + S22 @ T12 @ nS11
        nS22 = S22 @ T12 @ nS12 + S22 @ T11 @ d2
        S11, S12, S21, S22 = nS11, nS12, nS21, nS22

    i0 = order_index(0, 0, Mx, My)
    a0 = np.zeros(N2, dtype=np.complex128)
    a0[i0] = -complex(Ey0)
    a0[N + i0] = complex(Ex0)
    bN = np.zeros(N2, dtype=np.complex128)
    aN = S11 @ a0 + S12 @ bN
    b0 = S21 @ a0 + S22 @ bN

    def flux(ai, bi, reg):
        A = reg["kp"] @ reg["phi"] @ np.diag(1.0 / (omega * reg["q"]))
        pa, pb = reg["phi"] @ ai, reg["phi"] @ bi
        Aa, Ab = A @ ai, A @ bi
        diff = 0.5 * (np.conj(pb) * Aa - np.conj(Ab) * pa)
        fxy = (np.conj(Aa) * pa).real + diff
        bxy = -(np.conj(Ab) * pb).real + np.conj(diff)
        return fxy[:N] + fxy[N:], bxy[:N] + bxy[N:]

    fwd0, bwd0 = flux(a0, b0, R[0])
    fwdN, bwdN = flux(aN, bN, R[-1])
    norm = n_inc.real / math.cos(theta)

    def efield(ai, bi, reg):
        A = reg["kp"] @ reg["phi"] @ np.diag(1.0 / (omega * reg["q"]))
        return A @ (ai - bi)

    Esub = efield(aN, bN, R[-1])
    Einc = efield(a0, np.zeros(N2, dtype=np.complex128), R[0])
    ex_inc = Einc[N + i0]
    denom = ex_inc if abs(ex_inc) > 1e-30 else 1.0 + 0j
    sumR = float(np.sum((-bwd0).real * norm))
    sumT = float(np.sum(fwdN.real * norm))
    out = dict(R=sumR, T=sumT, sum_de=sumR + sumT, de_r0=float((-bwd0[i0]).real * norm),
               de_t0=float(fwdN[i0].real * norm), tx0=complex(Esub[N + i0] / denom),
               ty0=complex(-Esub[i0] / denom))
    if orders_out:
        k0sub = (n_sub.real * k0) ** 2
        k0inc = (n_inc.real * k0) ** 2
        kt2 = (kxv * kxv + kyv * kyv).real
        out["orders"] = [dict(p=int(p[i]), q=int(q[i]), de_t=float(fwdN[i].real * norm),
                              de_r=float((-bwd0[i]).real * norm), prop_t=bool(k0sub - kt2[i] > 0),
                              prop_r=bool(k0inc - kt2[i] > 0)) for i in range(N)]
    return out


def solve_cell(period_um=None, wavelength_um=None, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0,
               fill_x=0.5, fill_y=None, thickness_um=0.6, Mx=3, My=None, shape=RECT, shape_param=0.5,
               rotation_rad=0.0, grid=0, force_laurent=0, theta_rad=0.0, phi_rad=0.0, Ex0=1.0, Ey0=0.0,
               period_x_um=None, period_y_um=None, **_):
    """One-layer cell with the fields of celeris_rcwa_cell (include/celeris_b200.h)."""
    px = period_x_um if period_x_um is not None else period_um
    py = period_y_um if period_y_um is not None else period_um
    layer = dict(eps_pillar=eps_pillar, eps_bg=eps_bg, fill_x=fill_x,
                 fill_y=fill_x if fill_y is None else fill_y, thickness=thickness_um, shape=shape,
                 shape_param=shape_param, rotation=rotation_rad, grid=grid or None,
                 force_laurent=bool(force_laurent))
    return solve(n_inc, [layer], n_sub, px, py, wavelength_um, theta_rad, phi_rad, Ex0, Ey0, Mx,
                 Mx if My is None else My)


# ---- materials (constant / Sellmeier, src/celeris/materials/material.cpp:13-29) ----
def sellmeier_index(terms, wl):
    l2 = wl * wl
    n2 = 1.0 + sum(B * l2 / (l2 - C) for B, C in terms)
    return complex(math.sqrt(n2), 0.0)


FUSED_SILICA = [(0.6961663, 0.0684043 ** 2), (0.4079426, 0.1162414 ** 2), (0.8974794, 9.896161 ** 2)]
BK7 = [(1.03961212, 0.00600069867), (0.231792344, 0.0200179144), (1.01046945, 103.560653)]
