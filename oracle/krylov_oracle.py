"""CPU oracle for the Lanczos eigensolver (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs use
this module; the product path never does.

Restates the Hermitian ``KrylovKit.eigsolve`` (Lanczos) that the reference's
DMRG calls (``test_product_dmrg_state.jl:221-226``: krylovdim 3, maxiter 1,
which :SR).  KrylovKit is an absent dependency (an empty fork submodule), so
this follows its published algorithm (KrylovKit ``src/eigsolve/lanczos.jl``,
``src/factorizations/lanczos.jl``) on plain numpy vectors:

* initialise: beta0 = |x0|, v = x0/beta0, r = A x0/beta0, alpha = <x0, A x0>/beta0^2,
  r -= alpha v, then re-orthogonalise r against v while |r| < eta |r_prev|
  (ModifiedGramSchmidtIR, eta = 1/sqrt(2));
* expand: v' = r/beta, w = A v', alpha = <v', w>, w -= beta v, w -= alpha v',
  IR loop against v' with the reference norm sqrt(|w|^2 + alpha^2 + beta^2);
* process at K == krylovdim or beta <= tol: eigen-decompose the tridiagonal T,
  sort by the selector, f = beta U[K, :], count converged leading pairs;
* restart: keep (3 krylovdim + 2 converged) / 5 Ritz vectors and reduce
  [diag(D); f^T] to Lanczos form by bottom-up Householder reflections.

Parity status: unpinned against KrylovKit itself (no KrylovKit here); pinned
against exact diagonalisation where the Krylov space converges.
"""
from __future__ import annotations

import numpy as np

_EPS = float(np.finfo(np.float64).eps)


def _order(D, which):
    if which == "SR":
        return np.argsort(D, kind="stable")
    if which == "LR":
        return np.argsort(-D, kind="stable")
    if which == "SM":
        return np.argsort(np.abs(D), kind="stable")
    if which == "LM":
        return np.argsort(-np.abs(D), kind="stable")
    raise ValueError(which)


def householder_restore(D, f):
    """[diag(D); f^T] -> (alphas, betas, Q): Q^T diag(D) Q tridiagonal with
    diagonal alphas and off-diagonals betas[:-1]; f^T Q = betas[-1] e_k^T."""
    k = len(D)
    M = np.vstack([np.diag(np.asarray(D, dtype=float)), np.asarray(f, dtype=float)[None, :]])
    Q = np.eye(k)
    for col in reversed(range(k)):
        row = col + 1
        x = M[row, : col + 1].copy()
        n = np.sqrt(np.sum(x * x))
        if n == 0.0:
            continue
        nu = n if x[col] < 0 else -n
        u = x
        u[col] = u[col] - nu
        s = np.dot(u, u)
        if s == 0.0:
            continue
        P = np.eye(col + 1) - (2.0 / s) * np.outer(u, u)
        M[:, : col + 1] = M[:, : col + 1] @ P
        M[: col + 1, :] = P @ M[: col + 1, :]
        Q[:, : col + 1] = Q[:, : col + 1] @ P
        M[row, :col] = 0.0
        M[row, col] = nu
    return np.diag(M[:k, :k]).copy(), np.array([M[j + 1, j] for j in range(k)]), Q


def lanczos_eigsolve(matvec, x0, howmany=1, which="SR", krylovdim=30, maxiter=100, tol=1e-12,
                     eta=1.0 / np.sqrt(2.0)):
    """Returns (values, vectors, converged, numiter, numops) on numpy vectors."""
    x0 = np.asarray(x0, dtype=np.float64)
    b0 = np.linalg.norm(x0)
    Ax0 = matvec(x0)
    alpha = np.dot(x0, Ax0) / (b0 * b0)
    v = x0 / b0
    r = Ax0 / b0
    bold = np.linalg.norm(r)
    r = r - alpha * v
    beta = np.linalg.norm(r)
    while _EPS < beta < eta * bold:
        bold = beta
        d = np.dot(v, r)
        alpha += d
        r = r - d * v
        beta = np.linalg.norm(r)
    basis = [v]
    al, be = [alpha], [beta]
    nops, nit, conv = 1, 1, 0
    while True:
        beta = be[-1]
        K = len(basis)
        if beta <= tol and K < howmany:
            howmany = K
        if K == krylovdim or beta <= tol:
            T = np.diag(al) + np.diag(be[:-1], 1) + np.diag(be[:-1], -1)
            D, U = np.linalg.eigh(T)
            p = _order(D, which)
            D, U = D[p], U[:, p]
            f = beta * U[K - 1, :]
            conv = 0
            while conv < K and abs(f[conv]) <= tol:
                conv += 1
            if conv >= howmany:
                break
        if K < krylovdim:
            vn = r / beta
            basis.append(vn)
            w = matvec(vn)
            nops += 1
            a = np.dot(vn, w)
            w = w - beta * basis[-2]
            w = w - a * vn
            nrm = np.sqrt(a * a + beta * beta)
            b = np.linalg.norm(w)
            nold = np.sqrt(b * b + nrm * nrm)
            while _EPS < b < eta * nold:
                nold = b
                d = np.dot(vn, w)
                a += d
                w = w - d * vn
                b = np.linalg.norm(w)
            r = w
            al.append(a)
            be.append(b)
        else:
            if nit == maxiter:
                break
            keep = (3 * krylovdim + 2 * conv) // 5
            a2, b2, Q = householder_restore(D[:keep], f[:keep])
            B = np.stack(basis, axis=1) @ (U[:, :keep] @ Q)
            basis = [B[:, j].copy() for j in range(keep)]
            r = (b2[-1] / beta) * r
            al = list(a2)
            be = list(b2[:-1]) + [abs(b2[-1])]
            nit += 1
    if conv > howmany:
        howmany = conv
    Vm = np.stack(basis, axis=1)
    vecs = [Vm @ U[:, i] for i in range(howmany)]
    return list(D[:howmany]), vecs, conv, nit, nops
