"""End to end on a physical model: the spin-1/2 Heisenberg chain (J = 1, open
boundaries, U(1) conservation of 2Sz), N = 8, with the MPO of bond dimension 5
(I, S+, S-, Sz, I) stored as a U(1) block tensor.

The MPS has the exact (untruncated) bond dimensions, sector by sector.  Sites
left of the centre pair are random left isometries and sites right of it
random right isometries, so the two-site effective Hamiltonian at the centre is
the Hamiltonian of the 2Sz = 0 sector in another orthonormal basis.  On the GPU
the environments are built from the boundaries with make_L / make_R (the
contract! kernels), H_eff is applied by the four-contraction chain, and the
Lanczos eigensolver finds its lowest eigenvalue, which must equal the exact
ground-state energy of the chain (dense diagonalisation, 1e-10 relative).
H_eff·psi is also compared with a dense numpy contraction of the same tensors.
"""
import math

import numpy as np
import pytest

from sparsebackends_b200 import qn

pytestmark = pytest.mark.gpu

N = 8
PHYS = qn.PHYS  # 2Sz of s = 1 (up), 2 (down)


def bond_link(b):
    """Exact sector dimensions of bond b (b sites to its left), total 2Sz = 0."""
    charges, dims = [], []
    for q in range(-b, b + 1, 2):
        if abs(q) > N - b:
            continue
        left = math.comb(b, (b + q) // 2)
        right = math.comb(N - b, (N - b - q) // 2)
        charges.append(q)
        dims.append(min(left, right))
    return qn.U1Link(charges, dims)


# MPO channels: 1 = identity before, 2 = S+ placed (charge +2), 3 = S- placed
# (charge -2), 4 = Sz placed, 5 = identity after.  Link sectors: charge -2:
# [3], 0: [1, 4, 5], +2: [2] (channel -> (sector index 1-based, index in sector)).
MPO = qn.mpo_link({-2: 1, 0: 3, 2: 1})
CH = {1: (2, 1), 4: (2, 2), 5: (2, 3), 2: (3, 1), 3: (1, 1)}
SP = np.array([[0.0, 1.0], [0.0, 0.0]])  # <s'|S+|s>, s = 0 up, 1 down
SM = SP.T
SZ = np.diag([0.5, -0.5])
ID = np.eye(2)
TERMS = [(1, 1, ID), (5, 5, ID), (1, 2, SP), (2, 5, 0.5 * SM), (1, 3, SM), (3, 5, 0.5 * SP), (1, 4, SZ), (4, 5, SZ)]


def mpo_tensor(sb, ctx):
    """W[(qwl, s', s, qwr) | (mwl, mwr)] as a uniform block tensor."""
    blocks = {}
    for wl, wr, op in TERMS:
        (ql, ml), (qr, mr) = CH[wl], CH[wr]
        for sp in range(2):
            for s in range(2):
                if op[sp, s] == 0.0:
                    continue
                k = (ql, sp + 1, s + 1, qr)
                blk = blocks.setdefault(k, np.zeros((3, 3)))
                blk[ml - 1, mr - 1] += op[sp, s]
    keys = sorted(blocks, key=lambda k: (k[0] - 1) + 3 * ((k[1] - 1) + 2 * ((k[2] - 1) + 2 * (k[3] - 1))))
    data = np.concatenate([blocks[k].reshape(-1, order="F") for k in keys])
    return sb.NewBlockSparseSorted((3, 2, 2, 3, 3, 3), 2, keys, None, data, ctx=ctx), blocks


def isometry_site(rng, left, right, side):
    """Random site tensor A[(ql, s, qr) | ml, mr] (ragged triples), a left
    isometry (side 'L': sum over ql, ml, s of A^T A = I per qr) or a right one."""
    lay = qn.HeffLayout(left, right, MPO)
    keys = sorted(lay.keys["A"], key=lambda k: (k[0] - 1) + left.S * ((k[1] - 1) + 2 * (k[2] - 1)))
    blocks = {k: None for k in keys}
    if side == "L":
        for qr in range(1, right.S + 1):
            ks = [k for k in keys if k[2] == qr]
            rows = sum(left.dims[k[0] - 1] for k in ks)
            Q = np.linalg.qr(rng.standard_normal((rows, right.dims[qr - 1])))[0]
            o = 0
            for k in ks:
                r = left.dims[k[0] - 1]
                blocks[k] = Q[o:o + r]
                o += r
    else:
        for ql in range(1, left.S + 1):
            ks = [k for k in keys if k[0] == ql]
            cols = sum(right.dims[k[2] - 1] for k in ks)
            Q = np.linalg.qr(rng.standard_normal((cols, left.dims[ql - 1])))[0].T
            o = 0
            for k in ks:
                c = right.dims[k[2] - 1]
                blocks[k] = Q[:, o:o + c]
                o += c
    exts = [blocks[k].shape for k in keys]
    data = np.concatenate([blocks[k].reshape(-1, order="F") for k in keys])
    return lay, keys, data, exts, blocks


def dense_site(left, right, blocks):
    ol = np.concatenate([[0], np.cumsum(left.dims)[:-1]])
    orr = np.concatenate([[0], np.cumsum(right.dims)[:-1]])
    A = np.zeros((left.total, 2, right.total))
    for (ql, s, qr), b in blocks.items():
        A[ol[ql - 1]:ol[ql - 1] + b.shape[0], s - 1, orr[qr - 1]:orr[qr - 1] + b.shape[1]] = b
    return A


def exact_ground_energy():
    H = np.zeros((2 ** N, 2 ** N))
    for i in range(N - 1):
        for a, b, c in ((SZ, SZ, 1.0), (SP, SM, 0.5), (SM, SP, 0.5)):
            ops = [ID] * N
            ops[i], ops[i + 1] = a, b
            M = ops[0]
            for o in ops[1:]:
                M = np.kron(M, o)
            H += c * M
    # 2Sz = 0 sector: as many up (bit 0 of each site, state index 0) as down spins
    idx = [s for s in range(2 ** N) if bin(s).count("1") == N // 2]
    return float(np.linalg.eigvalsh(H[np.ix_(idx, idx)])[0])


def test_heisenberg_ground_energy_through_environments_and_lanczos():
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import krylov
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(7))
    bonds = [bond_link(b) for b in range(N + 1)]
    c = N // 2  # centre pair: sites c and c+1 (1-based), left bond c-1, right bond c+1
    W, wblocks = mpo_tensor(sb, ctx)
    Wd = np.zeros((5, 2, 2, 5))
    chan_index = {}
    oq = np.concatenate([[0], np.cumsum(MPO.dims)[:-1]])
    for ch, (q, m) in CH.items():
        chan_index[ch] = oq[q - 1] + m - 1
    for wl, wr, op in TERMS:
        Wd[chan_index[wl], :, :, chan_index[wr]] += op
    # boundary environments: bond 0 / bond N have one sector (charge 0, dim 1)
    q0 = MPO.index(0) + 1
    L = sb.NewBlockSparseSorted((1, 3, 1, 1, 3, 1), 3, [(1, q0, 1)], None, np.array([1.0, 0.0, 0.0]), ctx=ctx)
    R = sb.NewBlockSparseSorted((1, 3, 1, 1, 3, 1), 3, [(1, q0, 1)], None, np.array([0.0, 0.0, 1.0]), ctx=ctx)
    Ld = np.zeros((1, 5, 1))
    Ld[0, chan_index[1], 0] = 1.0
    Rd = np.zeros((1, 5, 1))
    Rd[0, chan_index[5], 0] = 1.0
    for i in range(1, c):  # sites 1 .. c-1, left isometries
        lay, keys, data, exts, blocks = isometry_site(rng, bonds[i - 1], bonds[i], "L")
        A = sb.NewBlockSparseSorted(lay.dims["A"], 2, keys, None, data, ctx=ctx, block_dims=exts)
        L = qn.make_L(L, A, W)
        Ad = dense_site(bonds[i - 1], bonds[i], blocks)
        Ld = np.einsum("xwa,asb,wtsv,xty->yvb", Ld, Ad, Wd, Ad)
    for i in range(N, c + 1, -1):  # sites N .. c+2, right isometries
        lay, keys, data, exts, blocks = isometry_site(rng, bonds[i - 1], bonds[i], "R")
        B = sb.NewBlockSparseSorted(lay.dims["A"], 2, keys, None, data, ctx=ctx, block_dims=exts)
        R = qn.make_R(R, B, W)
        Bd = dense_site(bonds[i - 1], bonds[i], blocks)
        Rd = np.einsum("ywb,asb,vtsw,xty->xva", Rd, Bd, Wd, Bd)
    # the centre two-site problem
    lay = qn.HeffLayout(bonds[c - 1], bonds[c + 1], MPO)
    pk, pdat, pe = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    psi = sb.NewBlockSparseSorted(lay.dims["psi"], 2, pk, None, pdat, ctx=ctx, block_dims=pe)
    op = qn.HeffOperator(lay, L, W, W, R, ctx)
    # H_eff psi against the dense contraction of the same environments
    hpsi = sb.to_dense(sb.to_uniform(op(psi)))
    from tests.heff_dense import _offsets
    ol, orr = _offsets(bonds[c - 1]), _offsets(bonds[c + 1])
    P = np.zeros((bonds[c - 1].total, 2, 2, bonds[c + 1].total))
    off = 0
    for (ql, s1, s2, qr), e in zip(pk, pe):
        n = int(np.prod(e))
        P[ol[ql - 1]:ol[ql - 1] + e[0], s1 - 1, s2 - 1, orr[qr - 1]:orr[qr - 1] + e[1]] = \
            pdat[off:off + n].reshape(e, order="F")
        off += n
    want = np.einsum("xwa,wpsv,vqtr,yrb,astb->xpqy", Ld, Wd, Wd, Rd, P)
    got = np.zeros_like(want)
    Dl, Dr = bonds[c - 1].D, bonds[c + 1].D
    for (ql, s1, s2, qr) in pk:
        el, er = bonds[c - 1].dims[ql - 1], bonds[c + 1].dims[qr - 1]
        got[ol[ql - 1]:ol[ql - 1] + el, s1 - 1, s2 - 1, orr[qr - 1]:orr[qr - 1] + er] = \
            hpsi[ql - 1, s1 - 1, s2 - 1, qr - 1, :el, :er]
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)
    # the lowest eigenvalue of H_eff is the exact ground-state energy
    vals, vecs, info = krylov.eigsolve(op, psi, 1, "SR", krylovdim=30, maxiter=100, tol=1e-11)
    e0 = exact_ground_energy()
    assert info.converged >= 1
    assert abs(vals[0] - e0) <= 1e-10 * abs(e0), (vals[0], e0)
