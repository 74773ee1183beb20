"""Callers of the far field on the GPU: through-focus and off-axis analyses of
the host mirror (celeris::analyze_through_focus, analyze_field_of_view,
analyze_wide_fov, analyze_field_grid; throughfocus.cpp:15-135, field.cpp) against
the reference's own CPU functions compiled into the oracle build, on a small
designed lens (f = 40 um, D = 16 um). The caustic (computed on the reference's
201 x 201 GPU grid) is checked against the oracle's x-z restatement.
"""
import math

import numpy as np
import pytest

from oracle import farfield as F

pytestmark = pytest.mark.gpu

F_UM, WL, D_UM = 40.0, 0.633, 16.0


def lens_and_lib():
    import celeris_b200 as cel

    lib = cel.UnitCellLibrary()
    lib.period_um, lib.wavelength_um, lib.thickness_um = 0.4, WL, 0.6
    nlib = 24
    lib.fill = list(np.linspace(0.2, 0.9, nlib))
    lib.phase = list(np.angle(np.exp(1j * np.linspace(0.0, 2 * np.pi, nlib, endpoint=False))))
    lib.amplitude = list(np.linspace(0.90, 0.97, nlib))
    lens = cel.design_metalens(lib, F_UM, D_UM)
    args = (lens.n_cells, lens.period_um, np.asarray(lens.fill_map), lib.fill, lib.phase, lib.amplitude,
            lib.wavelength_um)
    return cel, lib, lens, args


def test_through_focus_matches_reference():
    cel, lib, lens, args = lens_and_lib()
    tf = cel.analyze_through_focus(lens, lib, F_UM, WL, D_UM)
    z, I, zpk, dof = F.ref_through_focus(args, F_UM, WL, D_UM)
    assert np.array_equal(np.asarray(tf.z_um), z)
    assert np.max(np.abs(np.asarray(tf.intensity) - I)) <= 1e-6
    assert tf.z_peak_um == pytest.approx(zpk, abs=1e-6)
    assert tf.dof_um == pytest.approx(dof, abs=1e-5)
    # caustic: |E|^2 on the 201 x 201 x-z grid, normalized, vs the oracle
    n, p = lens.n_cells, lens.period_um
    c = (n - 1) / 2.0
    fm = np.asarray(lens.fill_map).reshape(n, n)
    px, py, t = [], [], []
    for iy in range(n):
        for ix in range(n):
            x, y = (ix - c) * p, (iy - c) * p
            if math.sqrt(x * x + y * y) > D_UM / 2:
                continue
            px.append(x)
            py.append(y)
            t.append(lib.transmission_for_fill(fm[iy, ix]))
    k = 2 * math.pi / WL
    Iz = F.rs_zx(np.array(px), np.array(py), np.array(t), tf.caustic_xmin, tf.caustic_xmax, 201, tf.caustic_zmin,
                 tf.caustic_zmax, 201, k)  # |E|^2, row = z
    Iz /= Iz.max()
    assert tf.caustic.shape == (201, 201)
    assert np.max(np.abs(np.asarray(tf.caustic) - Iz)) <= 1e-6


def test_field_of_view_matches_reference():
    cel, lib, lens, args = lens_and_lib()
    angles = [0.0, 2.0, 5.0, 9.0]
    got = cel.analyze_field_of_view(lens, lib, F_UM, WL, D_UM, angles)
    want = F.ref_field_of_view(args, F_UM, WL, D_UM, angles)
    for g, w in zip(got, want):
        assert g.angle_deg == w[0]
        assert g.rel_strehl == pytest.approx(w[1], rel=1e-9)
        assert g.spot_shift_um == pytest.approx(w[2], abs=1e-9)


def test_wide_fov_matches_reference():
    cel, lib, lens, args = lens_and_lib()
    angles = [0.0, 3.0, 6.0]
    got = cel.analyze_wide_fov(lens, lib, F_UM, WL, D_UM, 8.0, 20.0, angles)
    want = F.ref_wide_fov(args, F_UM, WL, D_UM, 8.0, 20.0, angles)
    for g, w in zip(got, want):
        assert g.rel_strehl == pytest.approx(w[1], rel=1e-9)
        assert g.spot_shift_um == pytest.approx(w[2], abs=1e-9)


def test_field_grid_matches_reference():
    cel, lib, lens, args = lens_and_lib()
    g = cel.analyze_field_grid(lens, lib, F_UM, WL, D_UM, 4.0, 1, 41)
    want = F.ref_field_grid(args, F_UM, WL, D_UM, 4.0, 1, 41)
    assert g.n == 3 and len(g.points) == 9
    for p, w in zip(g.points, want):
        got = [p.theta_x_deg, p.theta_y_deg, p.rel_strehl, p.fwhm_x_um, p.fwhm_y_um, p.cx_um, p.cy_um]
        assert got[:2] == list(w[:2])
        assert got[2] == pytest.approx(w[2], rel=1e-9)
        assert got[3:] == pytest.approx(list(w[3:]), abs=1e-9)


def test_chromatic_matches_reference():
    """analyze_chromatic (chromatic.cpp): 120-point on-axis scans per wavelength."""
    cel, lib, lens, args = lens_and_lib()
    got = cel.analyze_chromatic(lens, lib, F_UM, WL, D_UM, 0.5, 0.7, 5)
    want = F.ref_chromatic(args, F_UM, WL, D_UM, 0.5, 0.7, 5)
    for g, w in zip(got, want):
        assert g.wavelength_um == w[0]
        assert g.focal_length_um == pytest.approx(w[1], abs=1e-9)
        assert g.rel_peak == pytest.approx(w[2], rel=1e-9)


def test_chromatic_dispersive_with_per_wavelength_libraries():
    """analyze_chromatic_dispersive: with the same library at every wavelength it
    is analyze_chromatic of the reference; with a wavelength-dependent library
    (phases scaled by lambda0 / lambda) each scan is checked against the
    oracle's on-axis sum and the reference's first-maximum rule."""
    cel, lib, lens, args = lens_and_lib()
    got = cel.analyze_chromatic_dispersive(lens, lambda lam: lib, F_UM, WL, D_UM, 0.5, 0.7, 4)
    want = F.ref_chromatic(args, F_UM, WL, D_UM, 0.5, 0.7, 4)
    for g, w in zip(got, want):
        assert g.focal_length_um == pytest.approx(w[1], abs=1e-9)
        assert g.rel_peak == pytest.approx(w[2], rel=1e-9)

    def lib_at(lam):
        out = cel.UnitCellLibrary()
        out.period_um, out.wavelength_um, out.thickness_um = lib.period_um, lam, lib.thickness_um
        out.fill = list(lib.fill)
        out.phase = [float(np.angle(np.exp(1j * p * WL / lam))) for p in lib.phase]
        out.amplitude = list(lib.amplitude)
        return out

    got = cel.analyze_chromatic_dispersive(lens, lib_at, F_UM, WL, D_UM, 0.55, 0.7, 3)
    n, p = lens.n_cells, lens.period_um
    c = (n - 1) / 2.0
    fm = np.asarray(lens.fill_map).reshape(n, n)

    def cells(l):
        px, py, t = [], [], []
        for iy in range(n):
            for ix in range(n):
                x, y = (ix - c) * p, (iy - c) * p
                if math.sqrt(x * x + y * y) > D_UM / 2:
                    continue
                px.append(x)
                py.append(y)
                t.append(l.transmission_for_fill(fm[iy, ix]))
        return np.array(px), np.array(py), np.array(t)

    px, py, t = cells(lib_at(WL))
    k0 = 2 * math.pi / WL
    peak0 = F.rs_zx(px, py, t, 0.0, 0.0, 2, F_UM, F_UM, 2, k0)[0, 0]
    for g, lam in zip(got, [0.55, 0.625, 0.7]):
        px, py, t = cells(lib_at(lam))
        exp = F_UM * WL / lam
        I = F.rs_zx(px, py, t, 0.0, 0.0, 2, 0.55 * exp, 1.6 * exp, 120, 2 * math.pi / lam)[:, 0]
        j = int(np.argmax(I))  # first maximum, as the reference's strict > scan
        assert g.focal_length_um == pytest.approx(0.55 * exp + (1.6 * exp - 0.55 * exp) * j / 119, abs=1e-9)
        assert g.rel_peak == pytest.approx(I[j] / peak0, rel=1e-9)


def test_tolerance_monte_carlo_matches_reference():
    """analyze_tolerance (tolerance.cpp): same seeds, generator and normal
    distribution, each trial a focal analysis on the GPU."""
    cel, lib, lens, args = lens_and_lib()
    got = cel.analyze_tolerance(lens, lib, F_UM, WL, D_UM, [5.0, 25.0], 3, 7)
    want = F.ref_tolerance(args, F_UM, WL, D_UM, [5.0, 25.0], 3, 7)
    for g, w in zip(got, want):
        assert g.sigma_nm == w[0]
        assert [g.mean_strehl, g.worst_strehl] == pytest.approx([w[1], w[3]], rel=1e-6)
        assert g.std_strehl == pytest.approx(w[2], rel=1e-4, abs=1e-7)
