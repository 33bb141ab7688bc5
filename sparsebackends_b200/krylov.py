"""FP64 Lanczos eigensolver over device-resident block-sparse vectors.

This is the eigensolver the reference's DMRG calls through ITensorMPS:
``KrylovKit.eigsolve(PH, phi, 1, :SR; ishermitian=true, krylovdim=3,
maxiter=1, tol)`` (call sites ``test_product_dmrg_state.jl:221-226,258-259``;
``test_product.jl:235-238``).  Every vector operation runs on the GPU through
the library's vector-space hooks (``norm``, ``dot``, ``axpy!``, ``scale!``,
``copy``: ``src/tensor_wrappers.jl:793-923``); only the K x K tridiagonal
eigenproblem (K <= krylovdim) and scalar bookkeeping are host work, as in
KrylovKit.

KrylovKit itself is an absent dependency (its fork is an empty submodule at
``SparseBackends/Manifest.toml``); this follows its published Lanczos
algorithm (KrylovKit ``src/eigsolve/lanczos.jl`` and
``src/factorizations/lanczos.jl``):

* ``LanczosIterator`` with the default orthogonaliser ``ModifiedGramSchmidtIR``
  (eta = 1/sqrt(2)): three-term recurrence, then re-orthogonalisation against
  the newest basis vector while the residual norm drops below eta times its
  previous value;
* the factorisation is diagonalised when it reaches ``krylovdim`` (or the
  residual norm falls below ``tol``); Ritz values are sorted by ``which``
  (``"SR"``, ``"LR"``, ``"SM"``, ``"LM"``); Ritz pair i counts as converged while
  |beta * U[K, i]| <= tol, in order;
* restart (when ``maxiter`` > 1): keep (3 krylovdim + 2 converged) / 5 Ritz
  vectors and bring the projected matrix back to tridiagonal (Lanczos) form
  with Householder reflections from the bottom row up.

The operator ``A`` maps a vector to a new vector with the same block layout
(``qn.HeffOperator`` wraps the two-site H_eff chain that way).

Mixed precision: ``A`` may run its block GEMMs on the tensor cores (3xTF32,
``HeffOperator(..., precision="tf32x3")``) while every Lanczos vector,
inner product, norm and the tridiagonal eigenproblem stay FP64.  With
``correction`` (the same operator in FP64) each returned Ritz vector x gets
one FP64 apply: its value becomes the FP64 Rayleigh quotient <x, A x>/<x, x>
and ``info.residuals`` the FP64 residual norms |A x - E x| / |x|, so the
energy carries the tensor-core error only at second order in the vector's
error.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Tuple

import numpy as np

import sparsebackends_b200 as sb

EPS = float(np.finfo(np.float64).eps)
ETA = 1.0 / np.sqrt(2.0)

_SELECT = {
    "SR": (lambda d: d, False),
    "LR": (lambda d: d, True),
    "SM": (np.abs, False),
    "LM": (np.abs, True),
}


@dataclass
class ConvergenceInfo:
    converged: int
    normres: List[float]
    numiter: int
    numops: int
    residuals: list = field(default_factory=list)


def eigsort(D: np.ndarray, which: str) -> np.ndarray:
    """Permutation sorting Ritz values by the selector (stable, like sortperm)."""
    by, rev = _SELECT[which]
    key = by(D)
    return np.argsort(-key if rev else key, kind="stable")


def restore_lanczos_form(D: np.ndarray, f: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Householder reduction of the restarted projection back to Lanczos form.

    Input: the (k+1) x k matrix [diag(D); f^T] (kept Ritz values and their
    residual couplings).  Output (alphas, betas, Q) with Q orthogonal k x k,
    Q^T diag(D) Q = tridiag(betas[:-1], alphas, betas[:-1]) and f^T Q =
    betas[-1] e_k^T.  Rows are reduced from the bottom up (row j+1 over
    columns 0..j), as KrylovKit's restart does."""
    k = len(D)
    H = np.zeros((k + 1, k))
    H[np.arange(k), np.arange(k)] = D
    H[k, :] = f
    Q = np.eye(k)
    for j in range(k - 1, -1, -1):
        x = H[j + 1, : j + 1].copy()
        nx = np.linalg.norm(x)
        if nx == 0.0:
            continue
        nu = -nx if x[j] >= 0 else nx
        u = x.copy()
        u[j] -= nu
        uu = float(u @ u)
        if uu == 0.0:
            continue
        c = 2.0 / uu
        H[:, : j + 1] -= c * np.outer(H[:, : j + 1] @ u, u)
        H[: j + 1, :] -= c * np.outer(u, u @ H[: j + 1, :])
        Q[:, : j + 1] -= c * np.outer(Q[:, : j + 1] @ u, u)
        H[j + 1, :j] = 0.0
        H[j + 1, j] = nu
    alphas = np.array([H[j, j] for j in range(k)])
    betas = np.array([H[j + 1, j] for j in range(k)])
    return alphas, betas, Q


def _combine(V: List["sb._Tensor"], c: np.ndarray):
    """sum_i c[i] * V[i] as a new device vector."""
    t = sb.scale_(sb.copy(V[0]), float(c[0]))
    for i in range(1, len(V)):
        sb.axpy_(float(c[i]), V[i], t)
    return t


def eigsolve(A: Callable, x0, howmany: int = 1, which: str = "SR", *, krylovdim: int = 30, maxiter: int = 100,
             tol: float = 1e-12, eta: float = ETA, ishermitian: bool = True, correction: Callable = None,
             optol: float = 0.0):
    """``eigsolve(A, x0, howmany, which; ishermitian=true, krylovdim, maxiter, tol)``.

    Returns (values, vectors, info) like KrylovKit: ``values[i]`` and device
    tensors ``vectors[i]`` for the ``howmany`` selected Ritz pairs (more when
    more converged), and a ConvergenceInfo.  ``correction``: an FP64 operator
    for the residual correction of the returned pairs (module docstring).
    ``optol``: relative accuracy of ``A`` (0 for FP64); a new residual norm
    below ``optol`` times the largest recurrence coefficient so far is the
    operator's rounding noise, so the Krylov space counts as invariant, as a
    residual below ``tol`` does (a tensor-core operator on a space smaller
    than ``krylovdim`` would otherwise expand it with noise vectors)."""
    if not ishermitian:
        raise NotImplementedError("only the Hermitian (Lanczos) eigensolver is provided")
    if which not in _SELECT:
        raise ValueError(f"unknown selector {which!r}")
    if howmany > krylovdim:
        raise ValueError(f"krylov dimension {krylovdim} too small to compute {howmany} eigenvalues")

    # initialize (LanczosIterator)
    beta0 = sb.norm(x0)
    if beta0 == 0.0:
        raise ValueError("initial vector should not have norm zero")
    Ax0 = A(x0)
    alpha = sb.dot(x0, Ax0) / (beta0 * beta0)
    v = sb.scale_(sb.copy(x0), 1.0 / beta0)
    r = sb.scale_(Ax0, 1.0 / beta0)
    beta_old = sb.norm(r)
    sb.axpy_(-alpha, v, r)
    beta = sb.norm(r)
    while EPS < beta < eta * beta_old:
        beta_old = beta
        da = sb.dot(v, r)
        alpha += da
        sb.axpy_(-da, v, r)
        beta = sb.norm(r)
    V = [v]
    alphas, betas = [alpha], [beta]
    numops, numiter = 1, 1
    converged = 0
    D = U = f = None

    while True:
        beta = betas[-1]
        K = len(V)
        scale = max(max(abs(a) for a in alphas), max(betas))
        if optol > 0.0 and beta <= optol * scale:
            beta = 0.0  # numerically invariant for the operator's accuracy
        # a Ritz residual at the operator's noise level counts as converged:
        # restarting below it only mixes that noise into the basis
        ctol = max(tol, optol * scale)
        if beta <= tol and K < howmany:
            howmany = K
        if K == krylovdim or beta <= tol:
            T = np.diag(alphas) + np.diag(betas[:-1], 1) + np.diag(betas[:-1], -1)
            D, U = np.linalg.eigh(T)
            p = eigsort(D, which)
            D, U = D[p], U[:, p]
            f = beta * U[K - 1, :]
            converged = 0
            while converged < K and abs(f[converged]) <= ctol:
                converged += 1
            if converged >= howmany:
                break
        if K < krylovdim:
            # expand: v_{K+1} = r / beta, three-term recurrence plus IR
            vn = sb.scale_(r, 1.0 / beta)
            V.append(vn)
            w = A(vn)
            numops += 1
            a = sb.dot(vn, w)
            sb.axpy_(-beta, V[-2], w)
            sb.axpy_(-a, vn, w)
            ab2 = a * a + beta * beta
            b = sb.norm(w)
            nold = np.sqrt(b * b + ab2)
            while EPS < b < eta * nold:
                nold = b
                da = sb.dot(vn, w)
                a += da
                sb.axpy_(-da, vn, w)
                b = sb.norm(w)
            r = w
            alphas.append(a)
            betas.append(b)
        else:
            if numiter == maxiter:
                break
            keep = (3 * krylovdim + 2 * converged) // 5
            al, be, Q = restore_lanczos_form(D[:keep], f[:keep])
            M = U[:, :keep] @ Q
            V = [_combine(V, M[:, j]) for j in range(keep)]
            r = sb.scale_(r, float(be[-1]) / beta)  # residual nu * v_{K+1}
            alphas = [float(x) for x in al]
            betas = [float(x) for x in be[:-1]] + [abs(float(be[-1]))]
            numiter += 1

    if converged > howmany:
        howmany = converged
    values = [float(x) for x in D[:howmany]]
    vectors = [_combine(V, U[:, i]) for i in range(howmany)]
    normres = [abs(float(f[i])) for i in range(howmany)]
    info = ConvergenceInfo(converged, normres, numiter, numops)
    if correction is not None:
        for i, x in enumerate(vectors):
            y = correction(x)
            xx = sb.dot(x, x)
            e = sb.dot(x, y) / xx
            sb.axpy_(-e, x, y)
            info.residuals.append(float(np.sqrt(max(sb.dot(y, y), 0.0) / xx)))
            values[i] = float(e)
    return values, vectors, info
