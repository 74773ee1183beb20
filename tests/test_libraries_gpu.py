"""Library builders, designs and on-axis focus checks of the host mirror on the
GPU (celeris_b200/host/libraries.cpp) against the reference's OWN builder code
(design/achromatic.cpp, pb_achromatic.cpp, polar_metalens.cpp,
metalens.cpp:71-110) compiled into the oracle build, whose cell solves go to
the oracle's RCWA restatement. Library values within 1e-9 (phases, amplitudes)
and 1e-6 relative (group delays, least-squares slopes of those phases); designs
are given the same library on both sides and must pick the same atoms; focus
scans must find the same z sample and peak ratios within 1e-9.
"""
import math

import numpy as np
import pytest

from oracle import library as OL

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not OL.available(), reason="oracle/_ref not built")]

N_PIL, N_BG, N_INC, N_SUB = 2.4, 1.0, 1.0, 1.46
BAND = [0.50, 0.55, 0.60]
CENTER = 0.55


def mats(cel):
    c = cel.Material.constant
    return (c(complex(N_PIL), "pillar"), c(complex(N_BG), "bg"), c(complex(N_INC), "inc"), c(complex(N_SUB), "sub"))


def dphase(a, b):
    return abs((a - b + math.pi) % (2 * math.pi) - math.pi)


def check_dispersive(got, want_atoms, want_meta):
    assert got.center_index == int(want_meta[0])
    assert len(got.atoms) == len(want_atoms)
    for g, w in zip(got.atoms, want_atoms):
        assert dphase(g.phase0_rad, w["phase0"]) <= 1e-9
        assert g.mean_amplitude == pytest.approx(w["mean_amp"], abs=1e-9)
        assert g.group_delay_fs == pytest.approx(w["gd"], rel=1e-6, abs=1e-9)
        for j in range(len(BAND)):
            assert dphase(g.phase_rad[j], w["phase"][j]) <= 1e-9
            assert g.amplitude[j] == pytest.approx(w["amplitude"][j], abs=1e-9)
    assert got.gd_min_fs == pytest.approx(want_meta[1], rel=1e-6, abs=1e-9)
    assert got.gd_max_fs == pytest.approx(want_meta[2], rel=1e-6, abs=1e-9)


def test_dispersive_library_from_specs_four_shapes():
    import celeris_b200 as cel

    S = cel.MetaShape
    specs = [cel.MetaAtomSpec(S.Rectangle, 0.5, 0.5, 0.6, 0.5), cel.MetaAtomSpec(S.Ellipse, 0.6, 0.6, 0.6, 0.5),
             cel.MetaAtomSpec(S.Cross, 0.6, 0.6, 0.6, 0.5), cel.MetaAtomSpec(S.Ring, 0.7, 0.7, 0.6, 0.5)]
    got = cel.build_dispersive_library_from_specs(*mats(cel), 0.4, BAND, CENTER, specs, 3)
    want, meta = OL.dispersive_library_from_specs((N_PIL, N_BG, N_INC, N_SUB), 0.4, BAND, CENTER,
                                                  [(0, 0.5, 0.5, 0.6, 0.5), (1, 0.6, 0.6, 0.6, 0.5),
                                                   (2, 0.6, 0.6, 0.6, 0.5), (3, 0.7, 0.7, 0.6, 0.5)], 3)
    check_dispersive(got, want, meta)


def test_dispersive_library_fill_height_grid():
    import celeris_b200 as cel

    got = cel.build_dispersive_library(*mats(cel), 0.4, BAND, 0.56, 0.3, 0.8, 3, 0.5, 0.8, 2, 3)
    want, meta = OL.dispersive_library((N_PIL, N_BG, N_INC, N_SUB), 0.4, BAND, 0.56, 0.3, 0.8, 3, 0.5, 0.8, 2, 3)
    assert (got.n_fill, got.n_height) == (3, 2)
    check_dispersive(got, want, meta)
    assert [a.thickness_um for a in got.atoms] == [0.5] * 3 + [0.8] * 3


def test_single_etch_library_shape_families():
    import celeris_b200 as cel

    got = cel.build_single_etch_library(*mats(cel), 0.4, BAND[:2], 0.5, 0.4, 0.7, 2, 0.6, 2)
    specs = []
    for f in (0.4, 0.7):
        specs += [(0, f, f, 0.6, 0.5), (1, f, f, 0.6, 0.5)] + [(2, f, f, 0.6, a) for a in (0.3, 0.5, 0.7)] + \
                 [(3, f, f, 0.6, r) for r in (0.4, 0.6)]
    want, meta = OL.dispersive_library_from_specs((N_PIL, N_BG, N_INC, N_SUB), 0.4, BAND[:2], 0.5, specs, 2)
    assert len(got.atoms) == 14
    for g, w in zip(got.atoms, want):
        assert dphase(g.phase0_rad, w["phase0"]) <= 1e-9
        assert g.group_delay_fs == pytest.approx(w["gd"], rel=1e-6, abs=1e-9)


def test_dispersive_pb_library_filter_and_cross():
    import celeris_b200 as cel

    got = cel.build_dispersive_pb_library(*mats(cel), 0.4, BAND, CENTER, 0.25, 0.85, 3, 0.6, 3, 0.30)
    want, meta = OL.dispersive_pb_library((N_PIL, N_BG, N_INC, N_SUB), 0.4, BAND, CENTER, 0.25, 0.85, 3, 0.6, 3,
                                          0.30)
    assert len(got.atoms) == len(want) and 0 < len(want) < 9  # square pillars are filtered out
    for g, w in zip(got.atoms, want):
        assert (g.fill_x, g.fill_y) == (w["fill_x"], w["fill_y"])
        assert dphase(g.phase0_rad, w["phase0"]) <= 1e-9
        assert g.mean_amplitude == pytest.approx(w["mean_amp"], abs=1e-9)
        assert g.mean_conversion == pytest.approx(w["mean_conv"], abs=1e-9)
        assert g.retardance_center_deg == pytest.approx(w["retardance"], abs=1e-7)
        assert g.group_delay_fs == pytest.approx(w["gd"], rel=1e-6, abs=1e-9)
        assert np.max(np.abs(np.array(g.cross) - w["cross"])) <= 1e-9
    assert got.gd_min_fs == pytest.approx(meta[1], rel=1e-6, abs=1e-9)


def test_polarization_library_and_design():
    import celeris_b200 as cel

    got = cel.build_polarization_library(*mats(cel), 0.4, 0.633, 0.6, 0.25, 0.85, 4, 3)
    want = OL.polarization_library((N_PIL, N_BG, N_INC, N_SUB), 0.4, 0.633, 0.6, 0.25, 0.85, 4, 3)
    assert len(got.cells) == 16
    for g, w in zip(got.cells, want):
        assert (g.fill_x, g.fill_y) == (w[0], w[1])
        assert dphase(g.phase_x, w[2]) <= 1e-9 and dphase(g.phase_y, w[3]) <= 1e-9
        assert abs(g.amp_x - w[4]) <= 1e-9 and abs(g.amp_y - w[5]) <= 1e-9
    # design on the reference's library values, both sides
    lib = cel.PolarizationLibrary()
    lib.period_um, lib.wavelength_um, lib.thickness_um = 0.4, 0.633, 0.6
    cells = []
    for w in want:
        c = cel.PolarCell()
        c.fill_x, c.fill_y, c.phase_x, c.phase_y, c.amp_x, c.amp_y = (float(x) for x in w)
        cells.append(c)
    lib.cells = cells
    d = cel.design_polarization_metalens(lib, 30.0, 45.0, 12.0, 0.25)
    fills, metrics = OL.polarization_design(0.4, 0.633, want, 30.0, 45.0, 12.0, 0.25)
    assert np.array_equal(np.stack([d.fill_x, d.fill_y], axis=1), fills)
    assert [d.rms_phase_error_x_deg, d.rms_phase_error_y_deg, d.mean_amp_x, d.mean_amp_y] == \
        pytest.approx(list(metrics), rel=1e-12)


def test_unit_cell_library_stack():
    import celeris_b200 as cel

    c = cel.Material.constant
    air, sub = c(1.0 + 0j, "air"), c(complex(N_SUB), "sub")
    tio2, sio2 = c(2.4 + 0j, "TiO2"), c(1.46 + 0j, "SiO2")
    layers = [cel.RectCell2D(tio2, air, 0.5, 0.5, 0.5), cel.RectCell2D(sio2, air, 0.8, 0.8, 0.15)]
    got = cel.build_unit_cell_library_stack(cel.Rcwa2DStack(0.4, 0.4, layers), 0, air, sub, 0.633, 0.2, 0.8, 6, 3)
    fill, phase, amp = OL.unit_cell_library_stack([(2.4, 1.0, 0.5, 0.5, 0.5, 0, 0.5), (1.46, 1.0, 0.8, 0.8, 0.15, 0, 0.5)],
                                                  0.4, 0.4, 0, 1.0, N_SUB, 0.633, 0.2, 0.8, 6, 3)
    assert np.array_equal(np.asarray(got.fill), fill) and got.thickness_um == 0.5
    assert max(dphase(a, b) for a, b in zip(got.phase, phase)) <= 1e-9
    assert np.max(np.abs(np.asarray(got.amplitude) - amp)) <= 1e-9


def dispersive_for_design(cel):
    """A fill x height library with a usable group-delay range (GPU-built)."""
    return cel.build_dispersive_library(*mats(cel), 0.4, BAND, CENTER, 0.25, 0.85, 8, 0.5, 0.9, 3, 3)


def test_achromatic_design_and_focus_scan():
    import celeris_b200 as cel

    lib = dispersive_for_design(cel)
    f_um, d_um = 40.0, 16.0
    d = cel.design_achromatic_metalens(lib, f_um, d_um, 1.0, 0.25)
    focus = cel.verify_achromatic_focus(lib, d)
    rows = [[a.fill, a.thickness_um, a.phase0_rad, a.group_delay_fs, a.mean_amplitude, *a.phase_rad, *a.amplitude]
            for a in lib.atoms]
    idx, metrics, wf = OL.achromatic_design_verify(0.4, BAND, CENTER, lib.center_index, lib.gd_min_fs, lib.gd_max_fs,
                                                   rows, f_um, d_um, 1.0, 0.25)
    assert np.array_equal(np.asarray(d.atom_index), idx)
    got_m = [d.rms_phase_error_deg, d.rms_group_delay_error_fs, d.mean_amplitude, d.required_gd_span_fs,
             d.available_gd_span_fs, d.gd_coverage]
    assert got_m == pytest.approx(list(metrics), rel=1e-12)
    for g, w in zip(focus, wf):
        assert g.wavelength_um == w[0]
        assert g.focal_length_um == pytest.approx(w[1], abs=1e-9)
        assert g.rel_peak == pytest.approx(w[2], rel=1e-9)
    m = cel.to_metalens_design(d)
    assert m.n_cells == d.n_cells and np.array_equal(np.asarray(m.fill_map).ravel(), np.asarray(d.fill_map))


def test_pb_achromatic_design_and_focus_scan():
    import celeris_b200 as cel

    lib = cel.build_dispersive_pb_library(*mats(cel), 0.4, BAND, CENTER, 0.2, 0.85, 5, 0.6, 3, 0.2)
    f_um, d_um = 40.0, 16.0
    for hand in (1, -1):
        d = cel.design_pb_achromatic_metalens(lib, f_um, d_um, hand, 1.0, 0.25)
        focus = cel.verify_pb_achromatic_focus(lib, d)
        rows = []
        for a in lib.atoms:
            cr = np.array(a.cross)
            inter = np.empty(2 * len(cr))
            inter[0::2], inter[1::2] = cr.real, cr.imag
            rows.append([a.fill_x, a.fill_y, a.phase0_rad, a.group_delay_fs, a.mean_amplitude, a.mean_conversion,
                         *inter])
        idx, rot, metrics, wf = OL.pb_design_verify(0.4, 0.6, BAND, CENTER, lib.center_index, lib.gd_min_fs,
                                                    lib.gd_max_fs, rows, f_um, d_um, hand, 1.0, 0.25)
        assert np.array_equal(np.asarray(d.atom_index), idx)
        assert np.max(np.abs(np.asarray(d.rotation_rad) - rot)) <= 1e-12
        got_m = [d.rms_phase_error_deg, d.rms_group_delay_error_fs, d.mean_amplitude, d.mean_conversion,
                 d.gd_coverage]
        assert got_m == pytest.approx(list(metrics), rel=1e-9, abs=1e-9)
        for g, w in zip(focus, wf):
            assert g.focal_length_um == pytest.approx(w[1], abs=1e-9)
            assert g.rel_peak == pytest.approx(w[2], rel=1e-9)


def test_jones_hwp_atom_and_rotated_pb_check():
    """solve_jones, find_hwp_atom and verify_pb_phase (pb_metalens.cpp:36-104):
    the rotated atoms run the Laurent path with rotation, all in one batch."""
    import celeris_b200 as cel

    pil, bg, inc, sub = mats(cel)
    st = cel.Rcwa2DStack(0.4, 0.4, [cel.RectCell2D(pil, bg, 0.7, 0.3, 0.6)])
    J = cel.solve_jones(inc, st, sub, 0.633, 3)
    Jw = OL.solve_jones((N_PIL, N_BG, N_INC, N_SUB), 0.4, 0.7, 0.3, 0.6, 0.0, 0.633, 3)
    got = np.array([J.xx, J.xy, J.yx, J.yy])
    assert np.max(np.abs(got - Jw)) <= 1e-10 * np.max(np.abs(Jw))
    a = cel.find_hwp_atom(pil, bg, inc, sub, 0.4, 0.633, 0.6, 0.2, 0.8, 4, 3)
    aw = OL.find_hwp_atom((N_PIL, N_BG, N_INC, N_SUB), 0.4, 0.633, 0.6, 0.2, 0.8, 4, 3)
    assert a.conversion_efficiency == pytest.approx(aw["efficiency"], abs=1e-9)
    if (a.fill_x, a.fill_y) == (aw["fill_x"], aw["fill_y"]):
        assert abs(a.t_x - aw["t_x"]) <= 1e-9 and abs(a.t_y - aw["t_y"]) <= 1e-9
        assert a.retardance_deg == pytest.approx(aw["retardance"], abs=1e-7)
    else:
        # on a square period the atom and its x <-> y mirror image convert exactly
        # equally (|t_x - t_y| is symmetric), so the reference's first-maximum
        # rule (pb_metalens.cpp:57-72) meets an exact tie that rounding breaks
        assert (a.fill_x, a.fill_y) == (aw["fill_y"], aw["fill_x"])
        assert abs(a.t_x - aw["t_y"]) <= 1e-9 and abs(a.t_y - aw["t_x"]) <= 1e-9
        assert a.retardance_deg == pytest.approx(-aw["retardance"], abs=1e-7)
    rots = [0.0, 0.3, 0.7, 1.2]
    v = cel.verify_pb_phase(pil, bg, inc, sub, 0.4, 0.633, a, rots, 2)
    vw = OL.verify_pb_phase((N_PIL, N_BG, N_INC, N_SUB), 0.4, 0.633, a.fill_x, a.fill_y, 0.6, rots, 2)
    for g, w in zip(v, vw):
        assert g.rotation_deg == w[0]
        assert abs((g.cross_phase_deg - w[1] + 180) % 360 - 180) <= 1e-6
        assert g.conversion_eff == pytest.approx(w[2], abs=1e-9)
        assert g.copol_leakage == pytest.approx(w[3], abs=1e-9)
    # geometric-phase lens from the atom (host only)
    d = cel.design_pb_metalens(a, 0.4, 0.633, 20.0, 8.0, -1)
    rot, tc, met = OL.design_pb_metalens(a.t_x, a.t_y, 0.4, 0.633, 20.0, 8.0, -1)
    assert np.max(np.abs(np.asarray(d.rotation_rad) - rot)) <= 1e-12
    assert np.max(np.abs(np.asarray(d.t_cross) - tc)) <= 1e-12
    assert d.conversion_efficiency == pytest.approx(met[1], rel=1e-12)
    assert d.rms_phase_error_deg == pytest.approx(met[0], abs=1e-9)


def test_birefringence_sweep():
    import celeris_b200 as cel

    got = cel.analyze_birefringence(*mats(cel), 0.4, 0.633, 0.6, 0.35, 0.2, 0.8, 5, 3)
    want = OL.analyze_birefringence((N_PIL, N_BG, N_INC, N_SUB), 0.4, 0.633, 0.6, 0.35, 0.2, 0.8, 5, 3)
    for g, w in zip(got, want):
        assert (g.fill_x, g.fill_y) == (w[0], w[1])
        for a, b in ((g.phase_x_deg, w[2]), (g.phase_y_deg, w[3]), (g.retardance_deg, w[4])):
            assert abs((a - b + 180) % 360 - 180) <= 1e-6
        assert g.tx == pytest.approx(w[5], abs=1e-9) and g.ty == pytest.approx(w[6], abs=1e-9)


def test_optimize_system_grid():
    """optimize_system (system_opt.cpp): a 2 x 2 period x thickness grid, every
    library from one batched call, then design + focal analysis per point."""
    import celeris_b200 as cel

    calls = []
    got = cel.optimize_system(*mats(cel), 30.0, 10.0, 0.633, 0.35, 0.45, 0.5, 0.7, 2, 2, 12, 0.3,
                              lambda x: calls.append(x))
    want = OL.optimize_system((N_PIL, N_BG, N_INC, N_SUB), 30.0, 10.0, 0.633, 0.35, 0.45, 0.5, 0.7, 2, 2, 12, 0.3)
    assert (got.period_um, got.thickness_um) == (want[0], want[1])
    assert got.strehl == pytest.approx(want[2], rel=1e-6)
    assert got.mean_amplitude == pytest.approx(want[3], abs=1e-9)
    assert got.merit == pytest.approx(want[4], rel=1e-6)
    assert calls == pytest.approx([0.25, 0.5, 0.75, 1.0])
