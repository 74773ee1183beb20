"""The RCWA oracle (oracle/rcwa.py) pinned to the reference's own known answers
(cli/selftest.cpp case [8]): the subwavelength grating against the external
solver grcwa (TE 0.93334 within 2e-3, TM 0.96050 within 5e-3, M = 10),
energy conservation of the square TiO2 pillar across M, and the asymmetric
rectangular pillar against grcwa (0.954 / 0.972 within 0.03, M = 12). CPU only.
"""
import numpy as np
import pytest

from oracle import rcwa as RO

FS532 = RO.sellmeier_index(RO.FUSED_SILICA, 0.532)


def grating(Ex0, Ey0, M):
    layer = dict(eps_pillar=1.5 ** 2, eps_bg=1.0, fill_x=0.5, fill_y=1.0, thickness=0.5)
    return RO.solve(1.0, [layer], 1.0, 0.3, 0.3, 0.5, 0.0, 0.0, Ex0, Ey0, M, M)


def test_selftest8a_grating_vs_grcwa():
    te = grating(0.0, 1.0, 10)
    tm = grating(1.0, 0.0, 10)
    assert abs(te["de_t0"] - 0.93334) < 2e-3
    assert abs(tm["de_t0"] - 0.96050) < 5e-3


@pytest.mark.parametrize("M", [6, 8])
def test_selftest8b_square_pillar_energy(M):
    layer = dict(eps_pillar=2.45 ** 2, eps_bg=1.0, fill_x=0.5, fill_y=0.5, thickness=0.6)
    r = RO.solve(1.0, [layer], FS532, 0.35, 0.35, 0.532, 0.0, 0.0, 1.0, 0.0, M, M)
    assert abs(r["sum_de"] - 1.0) < 1e-4


@pytest.mark.timeout(600)
def test_selftest8c_rect_pillar_vs_grcwa():
    layer = dict(eps_pillar=2.45 ** 2, eps_bg=1.0, fill_x=0.6, fill_y=0.3, thickness=0.6)
    rx = RO.solve(1.0, [layer], FS532, 0.35, 0.35, 0.532, 0.0, 0.0, 1.0, 0.0, 12, 12)
    ry = RO.solve(1.0, [layer], FS532, 0.35, 0.35, 0.532, 0.0, 0.0, 0.0, 1.0, 12, 12)
    assert abs(rx["de_t0"] - 0.954) < 0.03 and abs(ry["de_t0"] - 0.972) < 0.03
    assert abs(rx["sum_de"] - 1.0) < 1e-4


def test_restatement_independent_of_the_eigensolver():
    """Eigenvector scaling and order are free (eig.hpp:16-18): the restatement
    with zgeev (scipy), with MKL's solver through torch on the CPU, and with the
    eigenvectors rescaled by random phases and magnitudes and permuted, gives the
    same cell to 1e-11."""
    import torch

    layer = dict(eps_pillar=2.45 ** 2, eps_bg=1.0, fill_x=0.6, fill_y=0.3, thickness=0.6)
    args = (1.0, [layer], FS532, 0.35, 0.35, 0.532, 0.1, 0.3, 0.6 + 0.2j, -0.3 + 0.7j, 4, 3)
    base = RO.solve(*args)

    def torch_eig(A):
        w, v = torch.linalg.eig(torch.tensor(A))
        return w.numpy(), v.numpy()

    rng = np.random.default_rng(5)

    def scrambled_eig(A):
        import scipy.linalg as sla

        w, v = sla.eig(A)
        perm = rng.permutation(len(w))
        scale = rng.uniform(0.5, 2.0, len(w)) * np.exp(1j * rng.uniform(0, 2 * np.pi, len(w)))
        return w[perm], (v * scale)[:, perm]

    for eig in (torch_eig, scrambled_eig):
        r = RO.solve(*args, eig=eig)
        for key in ("tx0", "ty0"):
            assert abs(r[key] - base[key]) <= 1e-11 * max(abs(base["tx0"]), abs(base["ty0"]))
        for key in ("R", "T", "de_t0", "de_r0"):
            assert abs(r[key] - base[key]) <= 1e-11
