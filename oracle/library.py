"""ORACLE - test infrastructure only (the checker).

ctypes access to oracle/_ref/libref_library.so: the REFERENCE's own library
builders, designs and on-axis focus checks (src/celeris/design/achromatic.cpp,
pb_achromatic.cpp, polar_metalens.cpp, pb_metalens.cpp, system_opt.cpp,
metalens.cpp:71-110, analysis/polarization.cpp) compiled from the reference tree
by oracle/Makefile. The reference's cell solve (rcwa2d.cpp) needs
Eigen, which is absent; the shim forwards every solve_rcwa_2d call to the numpy
restatement `oracle.rcwa.solve` through a callback registered here. So the
outputs are the reference's builder code over the oracle's cell solves.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from oracle import rcwa as RO

_HERE = os.path.dirname(os.path.abspath(__file__))
_PATH = os.path.join(_HERE, "_ref", "libref_library.so")
_lib = None

_P = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)
_CB = ctypes.CFUNCTYPE(ctypes.c_int, _P, ctypes.c_int, _P)


def _solve_cb(inp, nin, out):
    try:
        v = [inp[i] for i in range(nin)]
        n_inc, n_sub = complex(v[0], v[1]), complex(v[2], v[3])
        px, py, wl, th, ph = v[4:9]
        ex0, ey0 = complex(v[9], v[10]), complex(v[11], v[12])
        mx, my, nl = int(v[13]), int(v[14]), int(v[15])
        layers = []
        for l in range(nl):
            L = v[16 + 10 * l:26 + 10 * l]
            layers.append(dict(eps_pillar=complex(L[0], L[1]), eps_bg=complex(L[2], L[3]), fill_x=L[4],
                               fill_y=L[5], thickness=L[6], shape=int(L[7]), shape_param=L[8], rotation=L[9]))
        r = RO.solve(n_inc, layers, n_sub, px, py, wl, th, ph, ex0, ey0, mx, my)
        vals = [r["R"], r["T"], r["sum_de"], r["de_t0"], r["de_r0"], r["tx0"].real, r["tx0"].imag,
                r["ty0"].real, r["ty0"].imag]
        for i, x in enumerate(vals):
            out[i] = float(x)
        return 0
    except Exception:  # noqa: BLE001 - reported to the C++ side as a failed solve
        return 1


_cb_ref = _CB(_solve_cb)


def available() -> bool:
    return os.path.exists(_PATH)


def load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(_PATH)
        _lib.ref_set_rcwa_callback.argtypes = [_CB]
        _lib.ref_set_rcwa_callback(_cb_ref)
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_P)


def _mats(pillar, background, incident, substrate):
    return np.array([complex(pillar).real, complex(pillar).imag, complex(background).real,
                     complex(background).imag, complex(incident).real, complex(incident).imag,
                     complex(substrate).real, complex(substrate).imag])


def _unpack_dispersive(buf, n, nb):
    atoms = []
    for i in range(n):
        o = buf[i * (3 + 2 * nb):(i + 1) * (3 + 2 * nb)]
        atoms.append(dict(phase0=o[0], gd=o[1], mean_amp=o[2], phase=o[3:3 + nb].copy(),
                          amplitude=o[3 + nb:3 + 2 * nb].copy()))
    return atoms


def dispersive_library_from_specs(indices, period, band, center, specs, M):
    """specs: list of (shape, fill_x, fill_y, thickness, shape_param). Returns (atoms, meta)."""
    lib = load()
    mats, pm = _d(_mats(*indices))
    b, pb = _d(band)
    sp, psp = _d(np.array(specs, dtype=np.float64).ravel())
    nb, ns = len(band), len(specs)
    out = np.zeros(ns * (3 + 2 * nb))
    meta = np.zeros(3)
    lib.ref_build_dispersive_library_from_specs(pm, ctypes.c_double(period), pb, nb, ctypes.c_double(center), psp,
                                                ns, M, out.ctypes.data_as(_P), meta.ctypes.data_as(_P))
    return _unpack_dispersive(out, ns, nb), meta


def dispersive_library(indices, period, band, center, fill_min, fill_max, n_fills, thick_lo, thick_hi, n_heights, M):
    lib = load()
    mats, pm = _d(_mats(*indices))
    b, pb = _d(band)
    nb = len(band)
    out = np.zeros(max(1, n_fills * max(1, n_heights)) * (3 + 2 * nb))
    meta = np.zeros(3)
    f = ctypes.c_double
    n = lib.ref_build_dispersive_library(pm, f(period), pb, nb, f(center), f(fill_min), f(fill_max), n_fills,
                                         f(thick_lo), f(thick_hi), n_heights, M, out.ctypes.data_as(_P),
                                         meta.ctypes.data_as(_P))
    return _unpack_dispersive(out, n, nb), meta


def dispersive_pb_library(indices, period, band, center, fill_min, fill_max, n_fills, thickness, M, min_amplitude):
    lib = load()
    mats, pm = _d(_mats(*indices))
    b, pb = _d(band)
    nb = len(band)
    out = np.zeros(n_fills * n_fills * (7 + 2 * nb))
    meta = np.zeros(3)
    f = ctypes.c_double
    n = lib.ref_build_dispersive_pb_library(pm, f(period), pb, nb, f(center), f(fill_min), f(fill_max), n_fills,
                                            f(thickness), M, f(min_amplitude), out.ctypes.data_as(_P),
                                            meta.ctypes.data_as(_P))
    atoms = []
    for i in range(n):
        o = out[i * (7 + 2 * nb):(i + 1) * (7 + 2 * nb)]
        atoms.append(dict(fill_x=o[0], fill_y=o[1], phase0=o[2], gd=o[3], mean_amp=o[4], mean_conv=o[5],
                          retardance=o[6], cross=o[7::2][:nb] + 1j * o[8::2][:nb]))
    return atoms, meta


def polarization_library(indices, period, wavelength, thickness, fill_min, fill_max, n_samples, M):
    lib = load()
    mats, pm = _d(_mats(*indices))
    out = np.zeros(n_samples * n_samples * 6)
    f = ctypes.c_double
    n = lib.ref_build_polarization_library(pm, f(period), f(wavelength), f(thickness), f(fill_min), f(fill_max),
                                           n_samples, M, out.ctypes.data_as(_P))
    return out[:6 * n].reshape(n, 6)


def unit_cell_library_stack(layers, px, py, active, n_inc, n_sub, wavelength, fill_min, fill_max, n_samples, M):
    """layers: list of (pillar n, background n, fill_x, fill_y, thickness, shape, shape_param)."""
    lib = load()
    L = []
    for (npil, nbg, fx, fy, h, shape, sp) in layers:
        L += [complex(npil).real, complex(npil).imag, complex(nbg).real, complex(nbg).imag, fx, fy, h, shape, sp]
    Ld, pL = _d(L)
    ni, pni = _d([complex(n_inc).real, complex(n_inc).imag])
    ns, pns = _d([complex(n_sub).real, complex(n_sub).imag])
    fill, phase, amp = np.zeros(n_samples), np.zeros(n_samples), np.zeros(n_samples)
    f = ctypes.c_double
    lib.ref_build_unit_cell_library_stack(pL, len(layers), f(px), f(py), active, pni, pns, f(wavelength),
                                          f(fill_min), f(fill_max), n_samples, M, fill.ctypes.data_as(_P),
                                          phase.ctypes.data_as(_P), amp.ctypes.data_as(_P))
    return fill, phase, amp


def achromatic_design_verify(period, band, center, center_index, gd_min, gd_max, atoms, f_um, d_um, gd_weight,
                             amp_weight):
    """atoms: rows (fill, thickness, phase0, gd, mean_amp, phase[nb], amplitude[nb])."""
    lib = load()
    nb = len(band)
    b, pb = _d(band)
    A, pA = _d(np.asarray(atoms, dtype=np.float64).ravel())
    n = max(1, int(round(d_um / period)))
    idx = np.zeros(n * n, dtype=np.int32)
    metrics = np.zeros(6)
    focus = np.zeros(3 * nb)
    f = ctypes.c_double
    lib.ref_achromatic_design_verify(f(period), pb, nb, f(center), center_index, f(gd_min), f(gd_max), pA,
                                     len(atoms), f(f_um), f(d_um), f(gd_weight), f(amp_weight),
                                     idx.ctypes.data_as(_PI), metrics.ctypes.data_as(_P), focus.ctypes.data_as(_P))
    return idx, metrics, focus.reshape(nb, 3)


def pb_design_verify(period, thickness, band, center, center_index, gd_min, gd_max, atoms, f_um, d_um, handedness,
                     gd_weight, amp_weight):
    """atoms: rows (fill_x, fill_y, phase0, gd, mean_amp, mean_conv, cross re/im interleaved [2 nb])."""
    lib = load()
    nb = len(band)
    b, pb = _d(band)
    A, pA = _d(np.asarray(atoms, dtype=np.float64).ravel())
    n = max(1, int(round(d_um / period)))
    idx = np.zeros(n * n, dtype=np.int32)
    rot = np.zeros(n * n)
    metrics = np.zeros(5)
    focus = np.zeros(3 * nb)
    f = ctypes.c_double
    lib.ref_pb_design_verify(f(period), f(thickness), pb, nb, f(center), center_index, f(gd_min), f(gd_max), pA,
                             len(atoms), f(f_um), f(d_um), handedness, f(gd_weight), f(amp_weight),
                             idx.ctypes.data_as(_PI), rot.ctypes.data_as(_P), metrics.ctypes.data_as(_P),
                             focus.ctypes.data_as(_P))
    return idx, rot, metrics, focus.reshape(nb, 3)


def polarization_design(period, wavelength, cells, fx_um, fy_um, d_um, amp_weight):
    lib = load()
    C, pC = _d(np.asarray(cells, dtype=np.float64).ravel())
    n = max(1, int(round(d_um / period)))
    fills = np.zeros(2 * n * n)
    metrics = np.zeros(4)
    f = ctypes.c_double
    lib.ref_polarization_design(f(period), f(wavelength), pC, len(cells), f(fx_um), f(fy_um), f(d_um),
                                f(amp_weight), fills.ctypes.data_as(_P), metrics.ctypes.data_as(_P))
    return fills.reshape(n * n, 2), metrics


def solve_jones(indices, period, fill_x, fill_y, thickness, rotation, wavelength, M):
    lib = load()
    mats, pm = _d(_mats(*indices))
    out = np.zeros(8)
    f = ctypes.c_double
    lib.ref_solve_jones(pm, f(period), f(fill_x), f(fill_y), f(thickness), f(rotation), f(wavelength), M,
                        out.ctypes.data_as(_P))
    return out[0::2] + 1j * out[1::2]  # xx, xy, yx, yy


def find_hwp_atom(indices, period, wavelength, thickness, fill_min, fill_max, n_samples, M):
    lib = load()
    mats, pm = _d(_mats(*indices))
    out = np.zeros(9)
    f = ctypes.c_double
    lib.ref_find_hwp_atom(pm, f(period), f(wavelength), f(thickness), f(fill_min), f(fill_max), n_samples, M,
                          out.ctypes.data_as(_P))
    return dict(fill_x=out[0], fill_y=out[1], thickness=out[2], t_x=complex(out[3], out[4]),
                t_y=complex(out[5], out[6]), retardance=out[7], efficiency=out[8])


def verify_pb_phase(indices, period, wavelength, fill_x, fill_y, thickness, rotations, M):
    lib = load()
    mats, pm = _d(_mats(*indices))
    r, pr = _d(rotations)
    out = np.zeros(4 * len(rotations))
    f = ctypes.c_double
    lib.ref_verify_pb_phase(pm, f(period), f(wavelength), f(fill_x), f(fill_y), f(thickness), pr, len(rotations), M,
                            out.ctypes.data_as(_P))
    return out.reshape(-1, 4)


def design_pb_metalens(t_x, t_y, period, wavelength, f_um, d_um, handedness):
    lib = load()
    tx, ptx = _d([complex(t_x).real, complex(t_x).imag])
    ty, pty = _d([complex(t_y).real, complex(t_y).imag])
    n = max(1, int(round(d_um / period)))
    rot, tc, met = np.zeros(n * n), np.zeros(2 * n * n), np.zeros(2)
    f = ctypes.c_double
    lib.ref_design_pb_metalens(ptx, pty, f(period), f(wavelength), f(f_um), f(d_um), handedness,
                               rot.ctypes.data_as(_P), tc.ctypes.data_as(_P), met.ctypes.data_as(_P))
    return rot, tc[0::2] + 1j * tc[1::2], met


def analyze_birefringence(indices, period, wavelength, thickness, fill_y, fill_min, fill_max, n_samples, M):
    lib = load()
    mats, pm = _d(_mats(*indices))
    out = np.zeros(7 * n_samples)
    f = ctypes.c_double
    lib.ref_analyze_birefringence(pm, f(period), f(wavelength), f(thickness), f(fill_y), f(fill_min), f(fill_max),
                                  n_samples, M, out.ctypes.data_as(_P))
    return out.reshape(-1, 7)


def optimize_system(indices, f_um, d_um, wavelength, p_lo, p_hi, t_lo, t_hi, grid, M, fill_samples, eff_weight):
    lib = load()
    mats, pm = _d(_mats(*indices))
    out = np.zeros(5)
    f = ctypes.c_double
    lib.ref_optimize_system(pm, f(f_um), f(d_um), f(wavelength), f(p_lo), f(p_hi), f(t_lo), f(t_hi), grid, M,
                            fill_samples, f(eff_weight), out.ctypes.data_as(_P))
    return out


def optimize_pillar(indices, period, wavelength, target_phase, amplitude_weight, M, fill0, thickness0, max_iters):
    """The reference's optimize_pillar (optimize.cpp:22-86) over the oracle's cell
    solves. Returns dict(fill, thickness_um, phase, amplitude, loss, iterations)."""
    lib = load()
    mats, pm = _d(_mats(*indices))
    out = np.zeros(6)
    f = ctypes.c_double
    lib.ref_optimize_pillar(pm, f(period), f(wavelength), f(target_phase), f(amplitude_weight), M, f(fill0),
                            f(thickness0), max_iters, out.ctypes.data_as(_P))
    return dict(fill=out[0], thickness_um=out[1], phase=out[2], amplitude=out[3], loss=out[4],
                iterations=int(out[5]))
