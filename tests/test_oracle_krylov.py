"""CPU checks of the Lanczos oracle, the restart algebra and the vector hooks.

* the oracle Lanczos (restated KrylovKit eigsolve) converges to the exact
  lowest eigenpair of random symmetric matrices and of a Hermitian two-site
  H_eff, with and without restarts;
* the Householder restore of the restarted projection (oracle and the
  library's host-side copy) gives an orthogonal Q, a tridiagonal projection
  and a residual coupling on the last vector only;
* the oracle's vector hooks (norm, dot, x + y, map!) against dense numpy.
"""
import numpy as np
import pytest

from oracle import krylov_oracle as ko
from oracle import sparse_oracle as so
from sparsebackends_b200 import krylov, qn
from tests.heff_dense import heff_restricted, small_layout


def _sym(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    A = rng.standard_normal((n, n))
    return 0.5 * (A + A.T)


@pytest.mark.parametrize("restore", [ko.householder_restore, krylov.restore_lanczos_form])
@pytest.mark.parametrize("k,seed", [(1, 0), (2, 1), (5, 2), (9, 3)])
def test_householder_restore_gives_lanczos_form(restore, k, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    D = np.sort(rng.standard_normal(k))
    f = rng.standard_normal(k)
    a, b, Q = restore(D, f)
    assert np.allclose(Q.T @ Q, np.eye(k), atol=1e-13)
    T = Q.T @ np.diag(D) @ Q
    expect = np.diag(a) + np.diag(b[:-1], 1) + np.diag(b[:-1], -1)
    assert np.allclose(T, expect, atol=1e-12)
    g = f @ Q
    assert np.allclose(g[:-1], 0.0, atol=1e-12)
    assert abs(abs(g[-1]) - np.linalg.norm(f)) < 1e-12


@pytest.mark.parametrize("n,kdim,seed", [(60, 60, 4), (200, 12, 5), (300, 20, 6)])
def test_oracle_lanczos_converges_to_exact(n, kdim, seed):
    H = _sym(n, seed)
    x0 = np.random.Generator(np.random.PCG64(seed + 100)).standard_normal(n)
    vals, vecs, conv, nit, nops = ko.lanczos_eigsolve(lambda v: H @ v, x0, 1, "SR", krylovdim=kdim,
                                                      maxiter=500, tol=1e-10)
    ev, U = np.linalg.eigh(H)
    assert conv >= 1
    assert abs(vals[0] - ev[0]) <= 1e-9 * max(1.0, abs(ev[0]))
    v = vecs[0] / np.linalg.norm(vecs[0])
    assert min(np.linalg.norm(v - U[:, 0]), np.linalg.norm(v + U[:, 0])) < 1e-6


def test_oracle_lanczos_largest_and_smallest_magnitude():
    # positive definite, so the smallest-magnitude eigenvalue sits at the edge
    # of the spectrum (Lanczos without full re-orthogonalisation does not
    # resolve interior eigenvalues)
    H = _sym(80, 7)
    H += (abs(np.linalg.eigh(H)[0][0]) + 0.5) * np.eye(80)
    x0 = np.ones(80)
    ev = np.linalg.eigh(H)[0]
    for which, want in (("LR", ev[-1]), ("LM", ev[np.argmax(np.abs(ev))]), ("SM", ev[np.argmin(np.abs(ev))])):
        vals, *_ = ko.lanczos_eigsolve(lambda v: H @ v, x0, 1, which, krylovdim=80, maxiter=1, tol=1e-10)
        assert abs(vals[0] - want) < 1e-9


def test_oracle_lanczos_krylovdim3_maxiter1_is_one_pass():
    H = _sym(50, 8)
    x0 = np.random.Generator(np.random.PCG64(9)).standard_normal(50)
    vals, vecs, conv, nit, nops = ko.lanczos_eigsolve(lambda v: H @ v, x0, 1, "SR", krylovdim=3, maxiter=1,
                                                      tol=1e-14)
    assert (nit, nops) == (1, 3)
    # the Ritz value is the minimum of the Rayleigh quotient on span{x0, H x0, H^2 x0}
    Kb = np.linalg.qr(np.stack([x0, H @ x0, H @ (H @ x0)], axis=1))[0]
    assert abs(vals[0] - np.linalg.eigh(Kb.T @ H @ Kb)[0][0]) < 1e-10


def test_hermitian_heff_is_symmetric_and_oracle_finds_ground_state():
    lay = small_layout()
    rng = np.random.Generator(np.random.PCG64(11))
    ops = qn.hermitian_operators(lay, rng)
    keys, data, exts = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    H = heff_restricted(lay, ops, keys, exts)
    assert np.allclose(H, H.T, atol=1e-14)
    ev = np.linalg.eigh(H)[0]
    vals, *_ = ko.lanczos_eigsolve(lambda v: H @ v, data, 1, "SR", krylovdim=20, maxiter=300, tol=1e-11)
    assert abs(vals[0] - ev[0]) <= 1e-9 * max(1.0, abs(ev[0]))


def test_oracle_vector_hooks_against_dense():
    rng = np.random.Generator(np.random.PCG64(12))
    Ad = rng.standard_normal((4, 3, 5, 2)) * (rng.random((4, 3, 1, 1)) < 0.5)
    Bd = rng.standard_normal((4, 3, 5, 2)) * (rng.random((4, 3, 1, 1)) < 0.5)
    A, B = so.blocksparse_from_dense(Ad, 2), so.blocksparse_from_dense(Bd, 2)
    assert abs(so.bs_norm(A) - np.linalg.norm(Ad)) < 1e-12
    assert abs(so.bs_dot(A, B) - float(np.sum(Ad * Bd))) < 1e-12
    Cs = so.bs_add(A, B)
    assert np.array_equal(so.bs_to_dense(Cs), Ad + Bd)
    assert sorted(Cs.keys, key=lambda k: so.prefix_lin(k, (4, 3))) == Cs.keys
    assert set(Cs.keys) == set(A.keys) | set(B.keys)
    assert np.array_equal(so.bs_to_dense(so.bs_scale(-2.5, A)), -2.5 * Ad)
    r, a = rng.standard_normal(7), rng.standard_normal(7)
    assert np.array_equal(so.map_values("axpby", r, a, 0.3, -1.7), -1.7 * r + 0.3 * a)
    with pytest.raises(ValueError):
        so.map_values("axpy", r, a[:5])
