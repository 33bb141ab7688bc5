"""A dense einsum restatement of the PXP centre problem
(``sparsebackends_b200.pxp``), and converters from the oracle's block layout;
the oracle's own restatement is ``oracle.pxp_oracle``."""
import numpy as np

from oracle.pxp_oracle import OracleProblem, o_bs, o_contract, o_run  # noqa: F401
from sparsebackends_b200 import pxp


# ── dense restatement ───────────────────────────────────────────────────────

def dense_env_L(sites, c):
    """L[l', w, l] over sites 1..c-1 from the left boundary."""
    Wd = pxp.mpo_dense()
    L = np.zeros((1, pxp.W, 1))
    L[0, pxp.LEFT_CHANNEL - 1, 0] = 1.0
    for k in range(1, c):
        A = sites[k - 1]
        L = np.einsum("pwl,lsr,tswv,ptq->qvr", L, A, Wd, A, optimize=True)
    return L


def dense_env_R(sites, n, c):
    """R[r', w, r] over sites c+2..n from the right boundary."""
    Wd = pxp.mpo_dense()
    R = np.zeros((1, pxp.W, 1))
    R[0, pxp.RIGHT_CHANNEL - 1, 0] = 1.0
    for k in range(n, c + 1, -1):
        B = sites[k - 1]
        R = np.einsum("qvr,lsr,tswv,ptq->pwl", R, B, Wd, B, optimize=True)
    return R


def dense_heff(L, R, psi):
    Wd = pxp.mpo_dense()
    return np.einsum("pwl,labr,xawm,ybmv,qvr->pxyq", L, psi, Wd, Wd, R, optimize=True)


def env_to_dense(E, right: bool):
    """An oracle environment as E[m', w, m] (left layout (q', w, q | m', m),
    right layout (q', w, q | m, m'))."""
    d = E.dims
    m1, m2 = d[3], d[4]
    out = np.zeros((m2, d[1], m1) if right else (m1, d[1], m2))
    for k, i in zip(E.keys, E.ids):
        b = E.block(i).reshape(m1, m2, order="F")
        out[:, k[1] - 1, :] = b.T if right else b
    return out


def psi_to_dense(T):
    return pxp.psi_from_blocks(T.keys, np.concatenate([T.block(i) for i in T.ids]) if T.keys else np.zeros(0),
                               T.dims)
