"""CPU checks of the far-field oracle against the reference's golden vectors.

The golden fixtures (tests/golden/farfield_ref.npz) hold |E|^2 produced by the
reference's own celeris::propagate_pillars (focal.cpp:205-238); these tests pin
the plain-C restatement to them, and check the adjoint and caustic restatements
against dense numpy evaluations of the same formulas on small cases.
"""
import numpy as np
import pytest

from oracle import farfield as F

GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "farfield_ref.npz"))
CASES = sorted({k.split("/")[0] for k in GOLD.files})


def case(name):
    g = {k.split("/")[1]: GOLD[k] for k in GOLD.files if k.startswith(name + "/")}
    wl, z, cx, cy, n, W, k = g["params"]
    return g, float(wl), float(z), float(cx), float(cy), int(n), float(W), float(k)


@pytest.mark.parametrize("name", CASES)
def test_restatement_matches_reference_golden(name):
    g, wl, z, cx, cy, n, W, k = case(name)
    E = F.rs_field(g["px"], g["py"], g["t"], cx, cy, z, k, n, W)
    I = np.abs(E) ** 2
    assert np.max(np.abs(I - g["I_ref"])) <= 1e-13 * np.max(g["I_ref"])
    assert np.array_equal(E, g["E"])  # the restatement is deterministic


@pytest.mark.parametrize("name", CASES)
def test_reference_build_reproduces_golden(name):
    if F.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    g, wl, z, cx, cy, n, W, k = case(name)
    I = F.ref_propagate_pillars(g["px"], g["py"], g["t"], cx, cy, z, wl, n, W)
    assert np.array_equal(I, g["I_ref"])


def dense_G(px, py, cx, cy, z, k, n, W):
    step = 2.0 * W / (n - 1)
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    fx = (cx - W + i * step).reshape(-1, 1)
    fy = (cy - W + j * step).reshape(-1, 1)
    R = np.sqrt((fx - px[None]) ** 2 + (fy - py[None]) ** 2 + z * z)
    return np.exp(1j * k * R) / R


def test_pixels_subset_matches_full_grid():
    g, wl, z, cx, cy, n, W, k = case("offaxis_1000")
    idx = np.array([0, 5, n * n // 2, n * n - 1], dtype=np.int32)
    E = F.rs_pixels(g["px"], g["py"], g["t"], cx, cy, z, k, n, W, idx)
    assert np.array_equal(E, g["E"].reshape(-1)[idx])


def test_adjoint_is_conjugate_transpose():
    rng = np.random.default_rng(5)
    px, py = rng.uniform(-3, 3, 40), rng.uniform(-3, 3, 40)
    n, W, z, k = 7, 2.0, 20.0, 2 * np.pi / 0.6
    v = rng.normal(size=(n * n,)) + 1j * rng.normal(size=(n * n,))
    G = dense_G(px, py, 0.3, -0.1, z, k, n, W)
    out = F.rs_adjoint(px, py, 0.3, -0.1, z, k, n, W, v)
    ref = G.conj().T @ v
    assert np.max(np.abs(out - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_zx_matches_dense():
    rng = np.random.default_rng(6)
    px, py = rng.uniform(-3, 3, 30), rng.uniform(-3, 3, 30)
    t = rng.uniform(0.5, 1, 30) * np.exp(1j * rng.uniform(0, 6.3, 30))
    k = 2 * np.pi / 0.55
    out = F.rs_zx(px, py, t, -2.0, 2.0, 9, 15.0, 25.0, 6, k)
    fx = -2.0 + 4.0 * np.arange(9) / 8
    zz = 15.0 + 10.0 * np.arange(6) / 5
    R = np.sqrt((fx[None, :, None] - px) ** 2 + py ** 2 + zz[:, None, None] ** 2)
    E = (t * np.exp(1j * k * R) / R).sum(-1)
    assert np.max(np.abs(out - np.abs(E) ** 2)) <= 1e-12 * np.max(np.abs(E) ** 2)


def test_zero_pillars_and_single_pixel_grid():
    # npil == 0: zeros (focal.cpp:216). n == 1: step = 2W/0 = inf and 0*inf =
    # NaN, which the reference propagates (focal.cpp:223-227).
    E = F.rs_field(np.zeros(0), np.zeros(0), np.zeros(0, complex), 0, 0, 10.0, 1.0, 4, 1.0)
    assert np.all(E == 0)
    E1 = F.rs_field(np.array([0.0]), np.array([0.0]), np.array([1 + 0j]), 0, 0, 10.0, 1.0, 1, 1.0)
    assert np.isnan(E1[0, 0])
    if F.ref_lib() is not None:
        I1 = F.ref_propagate_pillars(np.array([0.0]), np.array([0.0]), np.array([1 + 0j]), 0, 0, 10.0, 1.0, 1, 1.0)
        assert np.isnan(I1[0, 0])
