"""The reference's own pass/fail checks (cli/selftest.cpp) for the RCWA callers,
run through the host mirror on the GPU: [12] form birefringence grows with
pillar asymmetry, [16] the Khorasaninejad 2016 nanofin is a near-ideal
half-wave plate with exact geometric phase, [20] efficiency budgets of a
lossless and an absorbing atom, [15] / [15b] / [15c] / [18] achromatic designs
(group-delay objective flattens the focal drift / lowers the group-delay RMS,
geometric phase exact, one etch). Materials are constant-index stand-ins where the
reference reads tabulated files (TiO2 2.45, SiO2 1.46, gold 0.54 + 2.2i at 532 nm).
"""
import math

import numpy as np
import pytest

import celeris_b200 as cel

pytestmark = pytest.mark.gpu


def test_selftest12_form_birefringence():
    tio2 = cel.Material.constant(2.40 + 0j, "TiO2~")
    air = cel.materials.air()
    retard = []
    for fx, fy in ((0.5, 0.5), (0.6, 0.4), (0.7, 0.3)):
        st = cel.Rcwa2DStack(0.35, 0.35, [cel.RectCell2D(tio2, air, fx, fy, 0.6)])
        J = cel.solve_jones(air, st, cel.materials.bk7(), 0.532, 8)
        d = (np.angle(J.xx) - np.angle(J.yy) + math.pi) % (2 * math.pi) - math.pi
        retard.append(abs(d) * 180 / math.pi)
    assert retard[0] < 1.0
    assert retard[2] > retard[1] > retard[0]
    # the same sweep through analyze_birefringence (fill_x swept at fixed fill_y)
    pts = cel.analyze_birefringence(tio2, air, air, cel.materials.bk7(), 0.35, 0.532, 0.6, 0.5, 0.5, 0.7, 3, 8)
    assert abs(pts[0].retardance_deg) < 1.0
    assert abs(pts[2].retardance_deg) > abs(pts[1].retardance_deg)


def test_selftest16_nanofin_half_wave_plate():
    tio2 = cel.Material.constant(2.45 + 0j, "TiO2~")
    air = cel.materials.air()
    U, H, lam = 0.325, 0.600, 0.532
    fx, fy = 0.095 / U, 0.250 / U
    st = cel.Rcwa2DStack(U, U, [cel.RectCell2D(tio2, air, fx, fy, H)])
    J = cel.solve_jones(air, st, cel.materials.fused_silica(), lam, 10)
    tx, ty = J.xx, J.yy
    T = 0.5 * (abs(tx) ** 2 + abs(ty) ** 2)
    conv_abs = abs(tx - ty) ** 2 / 4.0
    conv_rel = conv_abs / T
    retard = math.remainder(np.angle(tx) - np.angle(ty), 2 * math.pi) * 180 / math.pi
    atom = cel.HwpAtom()
    atom.fill_x, atom.fill_y, atom.thickness_um = fx, fy, H
    atom.t_x, atom.t_y, atom.conversion_efficiency = tx, ty, conv_abs
    d = cel.design_pb_metalens(atom, U, lam, 6.0, 6.0, 1)
    assert conv_rel > 0.95 and conv_rel > 0.73
    assert d.rms_phase_error_deg < 1e-6
    assert abs(abs(retard) - 180.0) < 15.0


def test_selftest20_efficiency_budget():
    air = cel.materials.air()
    tio2 = cel.Material.constant(2.45 + 0j, "TiO2")
    sio2 = cel.Material.constant(1.46 + 0j, "SiO2")
    au = cel.Material.constant(0.54 + 2.2j, "Au")
    bt = cel.analyze_efficiency(air, tio2, air, sio2, 0.35, 0.35, 0.6, 0.6, 0.6, 0.532, 1.0, 0.0, 6)
    assert abs(bt.transmission + bt.reflection + bt.absorption - 1.0) < 1e-3
    assert bt.absorption < 1e-3
    assert abs(bt.t_zero - bt.transmission) < 1e-4 and bt.n_prop_t == 1
    bg = cel.analyze_efficiency(air, au, air, sio2, 0.35, 0.35, 0.5, 0.5, 0.10, 0.532, 1.0, 0.0, 6)
    assert abs(bg.transmission + bg.reflection + bg.absorption - 1.0) < 1e-3 and bg.absorption > 0.2


BAND = [0.532 * 0.9, 0.532, 0.532 * 1.1]


def test_selftest15_achromatic_fill_height():
    """[15]: the group-delay objective flattens the chromatic focal drift while
    the base phase stays diffraction-limited."""
    tio2 = cel.Material.constant(2.40 + 0j, "TiO2~")
    air = cel.materials.air()
    dl = cel.build_dispersive_library(tio2, air, air, cel.materials.fused_silica(), 0.35, BAND, 0.532, 0.08, 0.92,
                                      10, 0.40, 1.40, 6, 5)
    sd = cel.design_achromatic_metalens(dl, 20.0, 6.0, 0.0)
    ad = cel.design_achromatic_metalens(dl, 20.0, 6.0, 1.0)

    def drift(c):
        z = [p.focal_length_um for p in c]
        return max(z) - min(z)

    assert drift(cel.verify_achromatic_focus(dl, ad)) < drift(cel.verify_achromatic_focus(dl, sd))
    assert ad.rms_phase_error_deg < 25.0


def test_selftest15b_single_etch():
    tio2 = cel.Material.constant(2.40 + 0j, "TiO2~")
    air = cel.materials.air()
    dl = cel.build_single_etch_library(tio2, air, air, cel.materials.fused_silica(), 0.35, BAND, 0.532, 0.08, 0.92,
                                       5, 0.80, 5)
    sd = cel.design_achromatic_metalens(dl, 20.0, 6.0, 0.0)
    ad = cel.design_achromatic_metalens(dl, 20.0, 6.0, 1.0)
    assert sd.single_height and ad.single_height
    assert ad.rms_group_delay_error_fs < sd.rms_group_delay_error_fs and ad.rms_phase_error_deg < 25.0


@pytest.mark.parametrize("case", ["15c", "18"])
def test_selftest15c_18_achromatic_pb(case):
    """[15c] / [18]: geometric base phase exact for both designs, group-delay RMS
    reduced by the group-delay objective, one etch depth."""
    tio2 = cel.Material.constant(2.40 + 0j, "TiO2~")
    air = cel.materials.air()
    if case == "15c":
        lib = cel.build_dispersive_pb_library(tio2, air, air, cel.materials.bk7(), 0.35, BAND, 0.532, 0.10, 0.90, 6,
                                              1.10, 5)
        f, D = 20.0, 6.0
    else:
        lib = cel.build_dispersive_pb_library(tio2, air, air, cel.materials.fused_silica(), 0.400,
                                              [0.470, 0.570, 0.670], 0.570, 0.10, 0.90, 6, 0.600, 5)
        f, D = 8.0, 5.0
    sd = cel.design_pb_achromatic_metalens(lib, f, D, 1, 0.0)
    ad = cel.design_pb_achromatic_metalens(lib, f, D, 1, 1.0)
    assert sd.rms_phase_error_deg < 1e-6 and ad.rms_phase_error_deg < 1e-6
    assert ad.rms_group_delay_error_fs < sd.rms_group_delay_error_fs
