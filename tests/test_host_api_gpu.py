"""The reference's Python surface (C++ host mirror `_celeris`) on the GPU.

Checks the drop-in calls against the oracle and against the reference's own
known answers: selftest [9] (cli/selftest.cpp:376-438: library phase coverage
> 300 deg, RMS phase error < 20 deg, FWHM within 0.1 um of lambda f / D,
Strehl > 0.5) and the reference's compiled propagate_pillars.
"""
import math

import numpy as np
import pytest

import celeris_b200 as cel
from oracle import farfield as F
from oracle import rcwa as RO

pytestmark = pytest.mark.gpu


def test_build_unit_cell_library_matches_oracle():
    n2 = cel.Material.constant(2.0 + 0j, "n2")
    sub = cel.Material.constant(1.46 + 0j, "sub")
    air = cel.materials.air()
    lib = cel.build_unit_cell_library(n2, air, air, sub, 0.4, 0.633, 0.6, 0.2, 0.9, 16, 3)
    assert len(lib.fill) == 16
    for i in (0, 5, 15):
        r = RO.solve_cell(period_um=0.4, wavelength_um=0.633, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0,
                          fill_x=lib.fill[i], thickness_um=0.6, Mx=3)
        t = lib.amplitude[i] * np.exp(1j * lib.phase[i])
        assert abs(t - r["tx0"]) <= 1e-10 * abs(r["tx0"])


def test_solve_rcwa_2d_reference_signature_and_errors():
    tio2 = cel.Material.constant(2.45 + 0j, "TiO2")
    air = cel.materials.air()
    fs = cel.materials.fused_silica()
    stack = cel.Rcwa2DStack(0.35, 0.35, [cel.RectCell2D(tio2, air, 0.5, 0.5, 0.6)])
    r = cel.solve_rcwa_2d(air, stack, fs, 0.532, 0.0, 0.0, 1.0, 0.0, 6, 6)
    assert abs(r.sum_de - 1.0) < 1e-4  # selftest [8b] (selftest.cpp:330-345)
    with pytest.raises(ValueError):
        cel.solve_rcwa_2d(air, stack, fs, 0.532, 0.0, 0.0, 1.0, 0.0, -1, 6)
    with pytest.raises(ValueError):
        cel.solve_rcwa_2d(air, cel.Rcwa2DStack(0.35, 0.35, []), fs, 0.532, 0.0, 0.0, 1.0, 0.0, 3, 3)


def test_solve_rcwa_2d_multilayer_stack():
    """Two patterned layers (a TiO2 pillar on a silica grating) through the
    reference's signature, against the oracle's multi-layer recursion."""
    tio2 = cel.Material.constant(2.45 + 0j, "TiO2")
    sio2 = cel.Material.constant(1.46 + 0j, "SiO2")
    air = cel.materials.air()
    sub = cel.Material.constant(1.46 + 0j, "sub")
    layers = [cel.RectCell2D(tio2, air, 0.5, 0.4, 0.45), cel.RectCell2D(sio2, air, 0.7, 0.7, 0.2)]
    stack = cel.Rcwa2DStack(0.35, 0.35, layers)
    r = cel.solve_rcwa_2d(air, stack, sub, 0.532, 0.0, 0.0, 1.0, 0.0, 3, 3)
    want = RO.solve(1.0, [dict(eps_pillar=2.45 ** 2, eps_bg=1.0, fill_x=0.5, fill_y=0.4, thickness=0.45),
                          dict(eps_pillar=1.46 ** 2, eps_bg=1.0, fill_x=0.7, fill_y=0.7, thickness=0.2)],
                    1.46, 0.35, 0.35, 0.532, 0.0, 0.0, 1.0, 0.0, 3, 3)
    assert abs(r.tx0 - want["tx0"]) <= 1e-10 * abs(want["tx0"])
    assert abs(r.R - want["R"]) <= 1e-10 and abs(r.T - want["T"]) <= 1e-10
    assert abs(r.sum_de - 1.0) <= 1e-10


def test_analyze_efficiency_budget():
    """analyze_efficiency (analysis/efficiency.cpp:7-46) on a lossy, diffracting
    meta-atom: the budget's sums and counts against the oracle's orders."""
    pil = cel.Material.constant(2.0 + 0.05j, "lossy")
    air = cel.materials.air()
    sub = cel.Material.constant(1.46 + 0j, "sub")
    b = cel.analyze_efficiency(air, pil, air, sub, 0.8, 0.8, 0.5, 0.5, 0.6, 0.633, 1.0, 0.0, 3)
    want = RO.solve(1.0, [dict(eps_pillar=(2.0 + 0.05j) ** 2, eps_bg=1.0, fill_x=0.5, fill_y=0.5, thickness=0.6)],
                    1.46, 0.8, 0.8, 0.633, 0.0, 0.0, 1.0, 0.0, 3, 3, orders_out=True)
    assert abs(b.reflection - want["R"]) <= 1e-10 and abs(b.transmission - want["T"]) <= 1e-10
    assert abs(b.absorption - max(0.0, 1 - want["R"] - want["T"])) <= 1e-10 and b.absorption > 1e-3
    assert abs(b.t_stray - max(0.0, want["T"] - want["de_t0"])) <= 1e-10
    assert b.n_prop_t == sum(o["prop_t"] for o in want["orders"])
    assert b.n_prop_r == sum(o["prop_r"] for o in want["orders"])
    de_t = [o.de_t for o in b.orders]
    assert de_t == sorted(de_t, reverse=True)
    assert abs(de_t[0] - max(o["de_t"] for o in want["orders"])) <= 1e-10


def test_selftest9_metalens_pipeline():
    tio2 = cel.Material.constant(2.40 + 0j, "TiO2~")
    air = cel.materials.air()
    lib = cel.build_unit_cell_library(tio2, air, air, cel.materials.bk7(), 0.35, 0.532, 0.6, 0.08, 0.92, 18, 6)
    assert lib.phase_span() * 180.0 / math.pi > 300.0
    lens = cel.design_metalens(lib, 50.0, 20.0)
    assert lens.rms_phase_error_deg < 20.0
    foc = cel.analyze_focus(lens, lib, 50.0, 0.532, 20.0)
    assert abs(foc.fwhm_um - foc.diffraction_limit_um) < 0.1
    assert foc.strehl > 0.5
    assert 0.0 < foc.encircled_energy <= 1.0
    # compute_psf equals the oracle field of the same aperture
    psf = cel.compute_psf(lens, lib, 50.0, 0.532, 20.0, 41, 3.0)
    n = lens.n_cells
    c = (n - 1) / 2.0
    fm = lens.fill_map
    px, py, t = [], [], []
    for iy in range(n):
        for ix in range(n):
            x, y = (ix - c) * lens.period_um, (iy - c) * lens.period_um
            if math.sqrt(x * x + y * y) > 10.0:
                continue
            px.append(x)
            py.append(y)
            t.append(lib.transmission_for_fill(fm[iy, ix]))
    E = F.rs_field(np.array(px), np.array(py), np.array(t), 0.0, 0.0, 50.0, 2 * math.pi / 0.532, 41, 3.0)
    I = np.abs(E) ** 2
    assert np.max(np.abs(psf.intensity - I)) <= 1e-10 * I.max()


def test_propagate_pillars_matches_reference_build():
    if F.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(4)
    px, py = rng.uniform(-6, 6, 500), rng.uniform(-6, 6, 500)
    t = rng.uniform(0.6, 1, 500) * np.exp(1j * rng.uniform(0, 6.3, 500))
    m = cel.propagate_pillars(list(px), list(py), list(t), 0.4, -0.2, 25.0, 0.55, 23, 2.0)
    ref = F.ref_propagate_pillars(px, py, t, 0.4, -0.2, 25.0, 0.55, 23, 2.0)
    assert np.max(np.abs(m.intensity - ref)) <= 1e-10 * ref.max()
    empty = cel.propagate_pillars([], [], [], 0.0, 0.0, 10.0, 0.5, 5, 1.0)
    assert np.all(empty.intensity == 0)


def test_optimize_pillar_reduces_loss():
    tio2 = cel.Material.constant(2.40 + 0j, "TiO2~")
    air = cel.materials.air()
    tgt = cel.PillarTarget(0.532, 1.0, 0.25)
    r0 = cel.optimize_pillar(tio2, air, air, cel.materials.fused_silica(), 0.35, tgt, 3, 0.5, 0.6, 0)
    r = cel.optimize_pillar(tio2, air, air, cel.materials.fused_silica(), 0.35, tgt, 3, 0.5, 0.6, 15)
    assert r.loss <= r0.loss
    assert 0.08 <= r.fill <= 0.92 and 0.2 <= r.thickness_um <= 1.0


@pytest.mark.parametrize("iters", [0, 1, 15])
def test_optimize_pillar_matches_reference_trajectory(iters):
    """optimize_pillar against the reference's own optimize.cpp:22-86 (central
    differences with h = 5e-3, Adam lr 0.04, box clamps), compiled into the
    oracle build with every cell solve forwarded to the oracle's RCWA: the same
    (fill, thickness, phase, |t|, loss) after 0, 1 and 15 steps."""
    from oracle import library as OL

    if not OL.available():
        pytest.skip("oracle/_ref not built")
    c = cel.Material.constant
    mats = (c(2.4 + 0j, "pillar"), c(1.0 + 0j, "bg"), c(1.0 + 0j, "inc"), c(1.46 + 0j, "sub"))
    tgt = cel.PillarTarget(0.532, 1.0, 0.25)
    got = cel.optimize_pillar(*mats, 0.35, tgt, 3, 0.5, 0.6, iters)
    want = OL.optimize_pillar((2.4, 1.0, 1.0, 1.46), 0.35, 0.532, 1.0, 0.25, 3, 0.5, 0.6, iters)
    assert got.iterations == want["iterations"] == iters
    assert abs(got.fill - want["fill"]) <= 1e-9
    assert abs(got.thickness_um - want["thickness_um"]) <= 1e-9
    assert abs(got.achieved_phase_rad - want["phase"]) <= 1e-9
    assert abs(got.achieved_amplitude - want["amplitude"]) <= 1e-9
    assert abs(got.loss - want["loss"]) <= 1e-9
