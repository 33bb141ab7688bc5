"""CPU oracle for the block factorisations (test infrastructure only).

Only ``tests/`` and the CPU legs of ``bench.py`` import this module; the
product path never does.

Restates ``SparseBackends/src/ops_factorize.jl`` with numpy's LAPACK-backed
``qr`` and ``svd`` (the reference calls LAPACK through Julia's LinearAlgebra):

* ``blocksparse_left_qr`` (ops_factorize.jl:8-43);
* ``blocksparse_svd`` (ops_factorize.jl:50-148), including the global
  truncation (stable decreasing sort of all singular values, keep
  min(maxdim, total), drop while count > mindim and sv < cutoff * max_sv).

Keys are 1-based tuples; blocks are flat column-major vectors.
"""
from __future__ import annotations

import numpy as np

from oracle.sparse_oracle import BS


def blocksparse_left_qr(A: BS):
    """Returns (Q: BS (l | s, b), R: ndarray k x n_r, l_vals, r_vals)."""
    assert A.N == 3 and A.n2 == 1
    l_vals = sorted({k[0] for k in A.keys})
    r_vals = sorted({k[1] for k in A.keys})
    li = {v: i for i, v in enumerate(l_vals)}
    ri = {v: i for i, v in enumerate(r_vals)}
    ds = A.dims[2]
    M = np.zeros((len(l_vals) * ds, len(r_vals)))
    for k, i in zip(A.keys, A.ids):
        a, b = li[k[0]], ri[k[1]]
        M[a * ds:(a + 1) * ds, b] = A.block(i)
    Qm, Rm = np.linalg.qr(M, mode="reduced")
    kk = min(M.shape)
    Qm, Rm = Qm[:, :kk], Rm[:kk, :]
    Q = BS.empty((A.dims[0], ds, kk), 2)
    for a, lv in enumerate(l_vals):
        blk = Qm[a * ds:(a + 1) * ds, :]
        bid = Q.ensure_block((lv,))
        Q.block(bid)[:] = blk.reshape(-1, order="F")
    return Q, Rm, l_vals, r_vals


def blocksparse_svd(A: BS, ortho="left", maxdim=2 ** 62, mindim=1, cutoff=0.0):
    """Returns (U: BS, SV: BS, svs_kept, (eigs, truncerr))."""
    assert A.N == 4 and A.n2 == 2
    nL, nR, d1, d2 = A.dims
    groups = {}
    for k in A.keys:
        groups.setdefault(k[0], []).append(k[1])
    blocks = A.blocks_by_key()
    svds = []
    for L in sorted(groups):
        rl = sorted(groups[L])
        Mi = np.zeros((d1, len(rl) * d2))
        for j, R in enumerate(rl):
            Mi[:, j * d2:(j + 1) * d2] = blocks[(L, R)].reshape((d1, d2), order="F")
        Ui, Si, Vti = np.linalg.svd(Mi, full_matrices=False)
        svds.append((L, Ui, Si, Vti, rl))
    allsv = [(float(s), bi, c) for bi, (_, _, Si, _, _) in enumerate(svds) for c, s in enumerate(Si)]
    allsv = sorted(allsv, key=lambda x: -x[0])  # stable, decreasing
    max_sv = allsv[0][0] if allsv else 1.0
    keep = min(maxdim, len(allsv))
    while keep > mindim and allsv[keep - 1][0] < cutoff * max_sv:
        keep -= 1
    truncerr = float(sum(x[0] ** 2 for x in allsv[keep:]))
    kk = [0] * len(svds)
    for i in range(keep):
        kk[allsv[i][1]] += 1
    nb = sum(kk)
    U = BS.empty((nL, max(nb, 1), d1), 1)
    U.dims = (nL, nb, d1)
    SV = BS.empty((max(nb, 1), nR, d2), 1)
    SV.dims = (nb, nR, d2)
    kept = np.zeros(nb)
    off = 0
    for bi, (L, Ui, Si, Vti, rl) in enumerate(svds):
        for col in range(kk[bi]):
            b = off + col + 1
            kept[b - 1] = Si[col]
            su = Si[col] if ortho == "right" else 1.0
            U.block(U.ensure_block((L, b)))[:] = Ui[:, col] * su
            sv = Si[col] if ortho == "left" else 1.0
            for j, R in enumerate(rl):
                SV.block(SV.ensure_block((b, R)))[:] = Vti[col, j * d2:(j + 1) * d2] * sv
        off += kk[bi]
    return U, SV, kept, (kept ** 2, truncerr)
