"""Dense two-site H_eff matrices for small U(1) layouts (test helper).

Builds the dense operators from the same seeded host blocks the device path
uploads, so the eigensolver tests can check against exact diagonalisation:
H[(a', s1', s2', b'), (a, s1, s2, b)] = sum_w L[a', wl, a] W1[wl, s1', s1, wm]
W2[wm, s2', s2, wr] R[b', wr, b], restricted to the psi blocks' entries in
payload order (the order of the ragged device vector)."""
from __future__ import annotations

import numpy as np

from sparsebackends_b200 import qn


def _offsets(link):
    return np.concatenate([[0], np.cumsum(link.dims)[:-1]]).astype(int)


def dense_from_ragged(layout, name, keys, data, exts):
    lab = layout.labels[name]
    P = len(lab) - layout.n2[name]
    ol, orr, ow = _offsets(layout.left), _offsets(layout.right), _offsets(layout.mpo)
    L_, R_, W_ = layout.left.total, layout.right.total, layout.mpo.total
    d = layout.d
    if name in ("L", "R"):
        o = ol if name == "L" else orr
        n = L_ if name == "L" else R_
        out = np.zeros((n, W_, n))
    elif name in ("W1", "W2"):
        out = np.zeros((W_, d, d, W_))
    else:  # psi
        out = np.zeros((L_, d, d, R_))
    off = 0
    for k, e in zip(keys, exts):
        cnt = int(np.prod(e))
        blk = data[off: off + cnt].reshape(e, order="F")
        off += cnt
        if name in ("L", "R"):
            qp, qw, q = k
            out[o[qp - 1]: o[qp - 1] + e[0], ow[qw - 1]: ow[qw - 1] + e[1], o[q - 1]: o[q - 1] + e[2]] = blk
        elif name in ("W1", "W2"):
            a, sp, s, b = k
            out[ow[a - 1]: ow[a - 1] + e[0], sp - 1, s - 1, ow[b - 1]: ow[b - 1] + e[1]] = blk
        else:
            ql, s1, s2, qr = k
            out[ol[ql - 1]: ol[ql - 1] + e[0], s1 - 1, s2 - 1, orr[qr - 1]: orr[qr - 1] + e[1]] = blk
    return out


def psi_indices(layout, keys, exts):
    """Flat (C-order over (a, s1, s2, b)) index of every psi payload entry."""
    ol, orr = _offsets(layout.left), _offsets(layout.right)
    shape = (layout.left.total, layout.d, layout.d, layout.right.total)
    idx = []
    for (ql, s1, s2, qr), (el, er) in zip(keys, exts):
        for mr in range(er):
            for ml in range(el):
                idx.append(np.ravel_multi_index((ol[ql - 1] + ml, s1 - 1, s2 - 1, orr[qr - 1] + mr), shape))
    return np.asarray(idx, dtype=np.int64)


def heff_restricted(layout, ops, psi_keys, psi_exts):
    """Dense H_eff restricted to the psi payload entries (payload order)."""
    L = dense_from_ragged(layout, "L", *ops["L"])
    W1 = dense_from_ragged(layout, "W1", *ops["W1"])
    W2 = dense_from_ragged(layout, "W2", *ops["W2"])
    R = dense_from_ragged(layout, "R", *ops["R"])
    H = np.einsum("xwa,wpsv,vqtr,yrb->xpqyastb", L, W1, W2, R, optimize=True)
    n = layout.left.total * layout.d * layout.d * layout.right.total
    H = H.reshape(n, n)
    idx = psi_indices(layout, psi_keys, psi_exts)
    return H[np.ix_(idx, idx)]


def small_layout(chi=24, charges=(-4, -2, 0, 2, 4), width=1.5, mpo=None):
    left = qn.gaussian_sectors(chi, list(charges), width=width)
    return qn.HeffLayout(left, left, qn.mpo_link(mpo or {-2: 2, 0: 3, 2: 2}))
