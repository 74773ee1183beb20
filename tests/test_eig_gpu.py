"""Standalone eigensolve (celeris_eig_general, the drop-in for eig.hpp:25) on
the GPU against LAPACK zgeev through numpy (the reference's CELERIS_USE_LAPACK
backend, eig.cpp:44-71): residual ||A V - V diag(lambda)|| / ||A|| <= 1e-12,
eigenvalues within 1e-10 ||A||, and for well-separated eigenvalues the
eigenvectors themselves (both unit-norm with the largest component real) within
1e-8.
"""
import numpy as np
import pytest

from celeris_b200 import capi

pytestmark = pytest.mark.gpu


def rand_matrix(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))


def match(vals, ref):
    """The permutation of the reference eigenvalues closest to the computed ones
    (an assignment, so repeated eigenvalues pair up one to one)."""
    from scipy.optimize import linear_sum_assignment

    rows, cols = linear_sum_assignment(np.abs(vals[:, None] - ref[None, :]))
    idx = np.empty(len(vals), dtype=int)
    idx[rows] = cols
    return idx


def check_pairs(A, vals, vecs, tol_vec=1e-8):
    nrm = np.linalg.norm(A, 2)
    assert np.linalg.norm(A @ vecs - vecs * vals) <= 1e-12 * nrm * max(1, A.shape[0]) ** 0.5
    assert np.allclose(np.linalg.norm(vecs, axis=0), 1.0, atol=1e-13)
    big = np.abs(vecs).argmax(axis=0)
    lead = vecs[big, np.arange(vecs.shape[1])]
    assert np.max(np.abs(lead.imag)) <= 1e-13 and np.all(lead.real > 0)
    rv, rV = np.linalg.eig(A)
    idx = match(vals, rv)
    assert np.max(np.abs(vals - rv[idx])) <= 1e-10 * nrm
    if tol_vec is not None:
        # zgeev's normalisation, same convention
        rV = rV[:, idx]
        bigr = np.abs(rV).argmax(axis=0)
        rV = rV * (np.abs(rV[bigr, np.arange(len(idx))]) / rV[bigr, np.arange(len(idx))])
        assert np.max(np.abs(vecs - rV)) <= tol_vec


@pytest.mark.parametrize("n", [2, 3, 17, 98, 113, 250])
def test_random_matrices_match_zgeev(n):
    A = rand_matrix(n, 100 + n)
    vals, vecs, info = capi.eig_general(A)
    assert info == 0
    check_pairs(A, vals, vecs)


def test_batch_equals_single_calls_and_order_one():
    As = np.stack([rand_matrix(40, s) for s in range(5)])
    vals, vecs, info = capi.eig_general(As)
    assert np.all(info == 0)
    for k in range(5):
        v1, V1, _ = capi.eig_general(As[k])
        assert np.array_equal(vals[k], v1) and np.array_equal(vecs[k], V1)
        check_pairs(As[k], vals[k], vecs[k])
    v, V, info = capi.eig_general(np.array([[2.5 - 1j]]))
    assert info == 0 and v[0] == 2.5 - 1j and V[0, 0] == 1.0


def test_degenerate_spectrum_residual():
    """Repeated eigenvalues (as symmetric unit cells give): eigenvectors are not
    unique, so only the residual and the eigenvalues are checked."""
    rng = np.random.default_rng(7)
    Q, _ = np.linalg.qr(rand_matrix(60, 8))
    d = np.repeat(rng.standard_normal(30) + 1j * rng.standard_normal(30), 2)
    A = Q @ np.diag(d) @ Q.conj().T
    vals, vecs, info = capi.eig_general(A)
    assert info == 0
    check_pairs(A, vals, vecs, tol_vec=None)


def test_host_mirror_signature():
    import celeris_b200 as cel

    A = rand_matrix(30, 3)
    vals, V = cel.eig_general(A)
    v2, V2, _ = capi.eig_general(A)
    assert np.array_equal(np.asarray(vals), v2) and np.array_equal(np.asarray(V), V2)


def test_reference_geev_batched_signature():
    """celeris::cuda::geev_batched (cuda/eigensolve.hpp:26-31): matrices column-major
    one after another, eigenvalues and right eigenvectors out; the reference's
    [10] check (eigenvalues of a 578 x 578 random matrix against the CPU solver)."""
    import celeris_b200 as cel

    rng = np.random.default_rng(42)
    A = rng.uniform(-1, 1, (578, 578)) + 1j * rng.uniform(-1, 1, (578, 578))
    As = np.stack([A.T, rand_matrix(578, 1).T])  # C-order of the transpose = column-major of A
    ok, w, vr = cel.cuda_geev_batched(As)
    assert ok
    ev = np.linalg.eigvals(A)
    assert np.max(np.abs(np.sort_complex(w[0]) - np.sort_complex(ev))) <= 1e-10 * np.linalg.norm(A, 2)
    V = vr[0].T  # back to row-major columns = eigenvectors
    assert np.linalg.norm(A @ V - V * w[0]) <= 1e-12 * np.linalg.norm(A, 2) * 578 ** 0.5
