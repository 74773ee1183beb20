"""Multi-layer RCWA stacks on the GPU, through the C ABI, against the oracle
restatement of solve_rcwa_2d with several layers (rcwa2d.cpp:209-488; the
S-matrix recursion of rcwa2d.cpp:376-401 over every interface): complex
order-0 transmission within 1e-10 relative, R and T within 1e-10, R + T = 1
for lossless stacks at normal incidence.
"""
import numpy as np
import pytest

from celeris_b200 import capi
from oracle import rcwa as RO

pytestmark = pytest.mark.gpu

TOL = 1e-10

COMMON = dict(period_um=0.4, wavelength_um=0.633, n_inc=1.0, n_sub=1.46)


def layer(**kw):
    d = dict(COMMON)
    d.update(eps_pillar=4.0, eps_bg=1.0, fill_x=0.5, thickness_um=0.3, Mx=3)
    d.update(kw)
    return d


def oracle_layer(c):
    return dict(eps_pillar=c["eps_pillar"], eps_bg=c["eps_bg"], fill_x=c["fill_x"],
                fill_y=c.get("fill_y", c["fill_x"]), thickness=c["thickness_um"],
                shape=c.get("shape", capi.SHAPE_RECT), shape_param=c.get("shape_param", 0.5),
                rotation=c.get("rotation_rad", 0.0), grid=c.get("grid", 0) or None,
                force_laurent=bool(c.get("force_laurent", 0)))


def ref(stack, Ex0, Ey0):
    c = stack[0]
    px = c.get("period_x_um", c.get("period_um"))
    py = c.get("period_y_um", c.get("period_um"))
    return RO.solve(c["n_inc"], [oracle_layer(x) for x in stack], c["n_sub"], px, py, c["wavelength_um"],
                    c.get("theta_rad", 0.0), c.get("phi_rad", 0.0), Ex0, Ey0, c["Mx"], c.get("My", c["Mx"]))


def check(got, want, lossless=True, power=1.0):
    scale = max(abs(want["tx0"]), abs(want["ty0"]))
    for key in ("tx0", "ty0"):
        assert abs(got[key] - want[key]) <= TOL * scale, (key, got[key], want[key])
    for key in ("R", "T", "de_t0", "de_r0"):
        assert abs(got[key] - want[key]) <= TOL, (key, got[key], want[key])
    if lossless:
        assert abs(got["R"] + got["T"] - power) <= TOL


STACKS = {
    # pillar on a patterned buffer layer
    "two_rect_M3": [layer(fill_x=0.55, thickness_um=0.6), layer(fill_x=0.8, eps_pillar=2.1, thickness_um=0.15)],
    # three layers, three Fourier rules (analytic rectangle, Laurent circle, asymmetric rectangle)
    "three_mixed_M3": [
        layer(fill_x=0.6, fill_y=0.35, thickness_um=0.25, eps_pillar=2.45 ** 2),
        layer(fill_x=0.6, thickness_um=0.4, eps_pillar=2.2 ** 2, shape=capi.SHAPE_ELLIPSE),
        layer(fill_x=0.45, thickness_um=0.2, eps_pillar=1.9 ** 2),
    ],
    # oblique incidence, rectangular period, M = (3, 2)
    "oblique_two_M32": [
        layer(period_x_um=0.45, period_y_um=0.38, theta_rad=0.15, phi_rad=0.4, Mx=3, My=2, fill_x=0.5,
              fill_y=0.6, thickness_um=0.35),
        layer(period_x_um=0.45, period_y_um=0.38, theta_rad=0.15, phi_rad=0.4, Mx=3, My=2, fill_x=0.7,
              thickness_um=0.2, eps_pillar=3.0, shape=capi.SHAPE_ELLIPSE),
    ],
    # absorbing top layer (lossy pillar)
    "lossy_two_M3": [layer(fill_x=0.5, thickness_um=0.1, eps_pillar=complex(-2.0, 1.5)),
                     layer(fill_x=0.6, thickness_um=0.5)],
}


def cells(stack):
    return [capi.rcwa_cell(**c) for c in stack]


@pytest.mark.parametrize("name", sorted(STACKS))
def test_stack_matches_oracle(name):
    stack = STACKS[name]
    # R + T = 1 only for lossless stacks at normal incidence: off normal the
    # reference's normalisation (n_inc / cos(theta), rcwa2d.cpp:437) of an
    # (Ex0, Ey0) excitation is not the incident power
    lossless = not name.startswith("lossy") and stack[0].get("theta_rad", 0.0) == 0.0
    res, info = capi.rcwa_stack_batch([cells(stack)])
    assert info[0] == 0
    check(res[0], ref(stack, 1.0, 0.0), lossless)
    check(res[1], ref(stack, 0.0, 1.0), lossless)


def test_single_stack_entry_complex_excitation():
    stack = STACKS["three_mixed_M3"]
    Ex0, Ey0 = 0.6 + 0.2j, -0.3 + 0.7j
    got = capi.solve_rcwa_2d_stack(cells(stack), Ex0, Ey0)
    want = ref(stack, Ex0, Ey0)
    check(got, want, power=abs(Ex0) ** 2 + abs(Ey0) ** 2)


def test_one_layer_stack_equals_batch():
    """A one-layer stack runs the plain recursion; the batch path the
    inverse-free second interface. Both must give the reference's answer."""
    c = layer(fill_x=0.55, thickness_um=0.6)
    s_res, s_info = capi.rcwa_stack_batch([cells([c])])
    b_res, b_info = capi.rcwa_batch(cells([c]))
    assert s_info[0] == 0 and b_info[0] == 0
    for k in range(2):
        check(s_res[k], b_res[k])


def test_uneven_stack_batch():
    """Stacks of 1-4 layers, two harmonic counts, in one call: results land in
    the caller's order."""
    rng = np.random.default_rng(3)
    batch = []
    for s in range(9):
        M = 2 if s % 3 == 0 else 3
        nl = 1 + s % 4
        batch.append([layer(Mx=M, fill_x=float(rng.uniform(0.3, 0.8)), thickness_um=float(rng.uniform(0.1, 0.4)),
                            shape=capi.SHAPE_ELLIPSE if (s + l) % 2 else capi.SHAPE_RECT) for l in range(nl)])
    res, info = capi.rcwa_stack_batch([cells(st) for st in batch])
    assert np.all(info == 0)
    for s in (0, 4, 7, 8):
        check(res[2 * s], ref(batch[s], 1.0, 0.0))
        check(res[2 * s + 1], ref(batch[s], 0.0, 1.0))


def test_stack_M5_blocked():
    """2N = 242: the blocked LU / GEMM paths of the recursion."""
    stack = [layer(Mx=5, fill_x=0.55, thickness_um=0.5), layer(Mx=5, fill_x=0.75, thickness_um=0.2, eps_pillar=2.5)]
    res, info = capi.rcwa_stack_batch([cells(stack)])
    assert info[0] == 0
    check(res[0], ref(stack, 1.0, 0.0))
    check(res[1], ref(stack, 0.0, 1.0))


@pytest.mark.parametrize("name", ["two_rect_M3", "oblique_two_M32"])
def test_orders_out_matches_oracle(name):
    """Per-order efficiencies (solve_rcwa_2d's orders_out, rcwa2d.cpp:464-485):
    labels and propagation flags exact, efficiencies within 1e-10."""
    stack = STACKS[name]
    c = stack[0]
    got, orders = capi.solve_rcwa_2d_orders(cells(stack), 1.0, 0.0)
    px = c.get("period_x_um", c.get("period_um"))
    py = c.get("period_y_um", c.get("period_um"))
    want = RO.solve(c["n_inc"], [oracle_layer(x) for x in stack], c["n_sub"], px, py, c["wavelength_um"],
                    c.get("theta_rad", 0.0), c.get("phi_rad", 0.0), 1.0, 0.0, c["Mx"], c.get("My", c["Mx"]),
                    orders_out=True)
    check(got, want, lossless=False)
    assert len(orders) == len(want["orders"])
    for g, w in zip(orders, want["orders"]):
        assert (g["p"], g["q"], g["prop_t"], g["prop_r"]) == (w["p"], w["q"], w["prop_t"], w["prop_r"])
        assert abs(g["de_t"] - w["de_t"]) <= TOL and abs(g["de_r"] - w["de_r"]) <= TOL
    assert abs(sum(o["de_t"] for o in orders) - got["T"]) <= TOL


def test_orders_one_layer_diffracting():
    """A period above the wavelength in the substrate (p = 0.9 um at 0.633 um):
    several orders propagate and carry power."""
    c = layer(period_um=0.9, fill_x=0.4, thickness_um=0.5)
    got, orders = capi.solve_rcwa_2d_orders(cells([c]), 0.0, 1.0)
    want = RO.solve(1.0, [oracle_layer(c)], 1.46, 0.9, 0.9, 0.633, 0.0, 0.0, 0.0, 1.0, 3, 3, orders_out=True)
    check(got, want)
    assert sum(o["prop_t"] for o in orders) > 1
    for g, w in zip(orders, want["orders"]):
        assert g["prop_t"] == w["prop_t"] and abs(g["de_t"] - w["de_t"]) <= TOL
