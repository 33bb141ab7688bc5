"""Two-site DMRG on the U(1) block format, the sweep of ITensorMPS ``dmrg``
(called by the reference's tests with krylovdim 3, maxiter 1 per bond:
``test_product_dmrg_state.jl:221-226``), run through the library's kernels.

Per bond (i, i+1) of a sweep: ψ = A_i·A_{i+1} (``contract!``), the lowest
eigenpair of the two-site H_eff by the device Lanczos (``krylov.eigsolve`` on
``qn.HeffOperator``), the U(1) split of the eigenvector
(``qn.split_two_site_device``, one GPU SVD per centre charge) into the new site tensors,
and the environment update (``qn.make_L`` / ``qn.make_R``).  Site tensors are
ragged block tensors A[(ql, s, qr) | (ml, mr)] in the "A" layout of
``qn.HeffLayout``; links are ``qn.U1Link`` with charge = 2Sz of the sites to
their left.  The MPO is the XXZ chain's (bond dimension 5: I, S+, S-, Sz, I)
with its link graded by the charge a channel carries.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np

from . import qn

SP = np.array([[0.0, 1.0], [0.0, 0.0]])  # <s'|S+|s>, s = 1 up, 2 down
SM = SP.T
SZ = np.diag([0.5, -0.5])
ID = np.eye(2)
# channels: 1 = identity before, 2 = S+ placed (carries +2), 3 = S- placed
# (-2), 4 = Sz placed, 5 = identity after; link sectors -2: [3], 0: [1, 4, 5],
# +2: [2] -> (1-based sector, index in the sector)
MPO_LINK = qn.mpo_link({-2: 1, 0: 3, 2: 1})
CHANNEL = {1: (2, 1), 4: (2, 2), 5: (2, 3), 2: (3, 1), 3: (1, 1)}


def xxz_terms(delta: float = 1.0):
    """(left channel, right channel, one-site operator) of H = Σ Sx Sx + Sy Sy + Δ Sz Sz."""
    return [(1, 1, ID), (5, 5, ID), (1, 2, SP), (2, 5, 0.5 * SM), (1, 3, SM), (3, 5, 0.5 * SP), (1, 4, SZ),
            (4, 5, delta * SZ)]


def mpo_blocks(delta: float = 1.0):
    """Host blocks of W[(qwl, s', s, qwr) | (mwl, mwr)]: key -> matrix at the
    key's channel-sector extents."""
    w = MPO_LINK
    blocks = {}
    for wl, wr, op in xxz_terms(delta):
        (ql, ml), (qr, mr) = CHANNEL[wl], CHANNEL[wr]
        for sp in range(2):
            for s in range(2):
                if op[sp, s] == 0.0:
                    continue
                k = (ql, sp + 1, s + 1, qr)
                blk = blocks.setdefault(k, np.zeros((w.dims[ql - 1], w.dims[qr - 1])))
                blk[ml - 1, mr - 1] += op[sp, s]
    return blocks


def mpo_tensor(ctx, delta: float = 1.0):
    """W[(qwl, s', s, qwr) | (mwl, mwr)], ragged (every block at its channel-sector extents)."""
    import sparsebackends_b200 as sb
    w = MPO_LINK
    blocks = mpo_blocks(delta)
    keys = sorted(blocks, key=lambda k: k[::-1])
    data = np.concatenate([blocks[k].reshape(-1, order="F") for k in keys])
    return sb.NewBlockSparseSorted((w.S, 2, 2, w.S, w.D, w.D), 2, keys, None, data, ctx=ctx,
                                   block_dims=[blocks[k].shape for k in keys])


def boundary_envs(ctx):
    """L0 holds the "identity before" channel, R0 the "identity after" one
    (both on the charge-0 channel sector; bond sectors of dimension 1)."""
    import sparsebackends_b200 as sb
    w = MPO_LINK
    q0 = w.index(0) + 1
    d0 = w.dims[q0 - 1]
    l0, r0 = np.zeros(d0), np.zeros(d0)
    l0[CHANNEL[1][1] - 1] = 1.0
    r0[CHANNEL[5][1] - 1] = 1.0
    dims = (1, w.S, 1, 1, w.D, 1)
    L = sb.NewBlockSparseSorted(dims, 3, [(1, q0, 1)], None, l0, ctx=ctx, block_dims=[(1, d0, 1)])
    R = sb.NewBlockSparseSorted(dims, 3, [(1, q0, 1)], None, r0, ctx=ctx, block_dims=[(1, d0, 1)])
    return L, R


def _site(ctx, left: qn.U1Link, right: qn.U1Link, keys, data, exts):
    import sparsebackends_b200 as sb
    return sb.NewBlockSparseSorted((left.S, 2, right.S, left.D, right.D), 2, keys, None, data, ctx=ctx,
                                   block_dims=exts)


def neel_state(ctx, n: int):
    """|up down up down ...> as site tensors with one 1x1 block each; bond b
    carries the charge of the first b sites."""
    bonds = [qn.U1Link([0], [1])]
    sites = []
    for i in range(n):
        s = 1 if i % 2 == 0 else 2
        bonds.append(qn.U1Link([bonds[-1].charges[0] + qn.PHYS[s - 1]], [1]))
        sites.append(_site(ctx, bonds[i], bonds[i + 1], [(1, s, 1)], np.ones(1), [(1, 1)]))
    return sites, bonds


DEVICE_SPLIT_ROWS = 48


def _host(t):
    return t.keys, np.array(t.data, copy=True), t.block_dims


class DMRG:
    """Two-site DMRG of the XXZ chain on ``n`` sites from the Néel state."""

    def __init__(self, n: int, delta: float = 1.0, ctx=None, precision: str = "f64", device_split="auto",
                 mpo=None, split_method: str = "svd"):
        """``precision``: the H_eff applies inside Lanczos run in that context
        precision ("tf32x3": tcgen05 3xTF32 with FP32 intermediates); the
        Lanczos vectors, orthogonalisation, the split and the environments stay
        FP64, and each bond's energy is the FP64 Rayleigh quotient of its Ritz
        vector (``krylov.eigsolve(..., correction=)``).  ``device_split``: True,
        the SVD per centre charge runs on the GPU (``qn.split_two_site_device``);
        False, the host numpy split; "auto", the GPU for bonds whose largest
        centre-charge matrix has at least ``DEVICE_SPLIT_ROWS`` rows (below
        that the launches of the device path cost more than the work).
        ``mpo``: a site-dependent MPO (``j1j2.J1J2Cylinder``: ``link``,
        ``tensors(ctx)``, ``boundary_envs(ctx)``) instead of the XXZ chain's;
        ``delta`` is then unused.  ``split_method``: the device split's
        factorisation, "svd" or "gram" (``qn.split_two_site_device``)."""
        import sparsebackends_b200 as sb
        self.sb = sb
        self.ctx = ctx or sb.default_context()
        self.precision = precision
        # Lanczos breakdown threshold (krylov.eigsolve's optol) of the sweeps:
        # a new direction below it counts as the operator's rounding.  The
        # sweeps refine every bond again, so it sits below the operator's
        # per-apply accuracy: on the N = 100 Heisenberg chain (chi to 109) 1e-7
        # gives the FP64 energy to 1.7e-11, 1e-6 to 4.8e-10, 1e-5 to 2.3e-8
        # (bonds whose residual falls below it stop improving)
        self.optol = {"f64": 0.0, "tf32x3": 1e-7, "tf32": 3e-2}[precision]
        self.device_split = device_split
        self.split_method = split_method
        self.n = n
        if mpo is None:
            self.mpo_link = MPO_LINK
            self.Ws = [mpo_tensor(self.ctx, delta)] * n
            L0, R0 = boundary_envs(self.ctx)
        else:
            self.mpo_link = mpo.link
            self.Ws = mpo.tensors(self.ctx)
            L0, R0 = mpo.boundary_envs(self.ctx)
        self.sites, self.bonds = neel_state(self.ctx, n)
        # Lenv[b]: sites 1..b, Renv[b]: sites b+1..n
        self.Lenv: List = [None] * (n + 1)
        self.Renv: List = [None] * (n + 1)
        self.Lenv[0], self.Renv[n] = L0, R0
        for b in range(n - 1, 0, -1):
            self.Renv[b] = qn.make_R(self.Renv[b + 1], self.sites[b], self.Ws[b])
        self.energy: Optional[float] = None
        self.truncerr = 0.0

    def _two_site(self, i: int):
        """ψ of bond (i, i+1) (1-based sites) on every charge-allowed key."""
        sb = self.sb
        A, B = self.sites[i - 1], self.sites[i]
        psi = qn.contract_new(["ql", "s1", "s2", "qr", "ml", "mr"], 2, A, ["ql", "s1", "qc", "ml", "mc"],
                              B, ["qc", "s2", "qr", "mc", "mr"])
        lay = qn.HeffLayout(self.bonds[i - 1], self.bonds[i + 1], self.mpo_link)
        keys = sorted(lay.keys["psi"], key=lambda k: k[::-1])
        exts = [lay.valid_extent("psi", k) for k in keys]
        if psi.keys == keys and [tuple(e) for e in psi.block_dims] == [tuple(e) for e in exts]:
            return lay, psi  # every allowed block already there, at its extents
        have = psi.blocks_by_key()
        parts = [have[k] if k in have else np.zeros(int(np.prod(e))) for k, e in zip(keys, exts)]
        data = np.concatenate(parts) if parts else np.zeros(0)
        x = sb.NewBlockSparseSorted(lay.dims["psi"], 2, keys, None, data, ctx=self.ctx, block_dims=exts)
        return lay, x

    def _update(self, i: int, absorb: str, maxdim: int, cutoff: float, krylovdim: int, maxiter: int):
        from . import krylov
        lay, x = self._two_site(i)
        ops = (lay, self.Lenv[i - 1], self.Ws[i - 1], self.Ws[i], self.Renv[i + 1], self.ctx)
        op = qn.HeffOperator(*ops, precision=self.precision)
        corr = qn.HeffOperator(*ops) if self.precision != "f64" else None
        vals, vecs, _ = krylov.eigsolve(op, x, 1, "SR", krylovdim=krylovdim, maxiter=maxiter, tol=1e-14,
                                        correction=corr, optol=self.optol)
        self.energy = float(vals[0])
        on_device = self.device_split
        if on_device == "auto":
            rows = {}
            for (ql, s1, s2, qr) in lay.keys["psi"]:
                c = lay.left.charges[ql - 1] + qn.PHYS[s1 - 1]
                rows.setdefault(c, set()).add((ql, s1))
            on_device = max(sum(lay.left.dims[ql - 1] for ql, _ in r) for r in rows.values()) >= DEVICE_SPLIT_ROWS
        if on_device:
            A, B, link, _, err = qn.split_two_site_device(lay, vecs[0], maxdim=maxdim, cutoff=cutoff, absorb=absorb,
                                                          method=self.split_method)
        else:
            (ak, ad, ae), (bk, bd, be), link, _, err = qn.split_two_site(lay, *_host(vecs[0]), maxdim=maxdim,
                                                                       cutoff=cutoff, absorb=absorb)
            A = _site(self.ctx, self.bonds[i - 1], link, ak, ad, ae)
            B = _site(self.ctx, link, self.bonds[i + 1], bk, bd, be)
        self.truncerr = max(self.truncerr, err)
        self.bonds[i] = link
        self.sites[i - 1] = A
        self.sites[i] = B

    def sweep(self, maxdim: int, cutoff: float = 0.0, krylovdim: int = 3, maxiter: int = 1) -> float:
        """One left-to-right and one right-to-left pass; returns the last energy."""
        n = self.n
        for i in range(1, n):
            self._update(i, "right", maxdim, cutoff, krylovdim, maxiter)
            self.Lenv[i] = qn.make_L(self.Lenv[i - 1], self.sites[i - 1], self.Ws[i - 1])
        for i in range(n - 1, 0, -1):
            self._update(i, "left", maxdim, cutoff, krylovdim, maxiter)
            self.Renv[i] = qn.make_R(self.Renv[i + 1], self.sites[i], self.Ws[i])
        return self.energy

    def run(self, maxdims: List[int], cutoff: float = 0.0, krylovdim: int = 3, maxiter: int = 1) -> Tuple[float, list]:
        energies = [self.sweep(m, cutoff, krylovdim, maxiter) for m in maxdims]
        return energies[-1], energies


def exact_ground_energy(n: int, delta: float = 1.0) -> float:
    """Lowest eigenvalue of the XXZ chain in the total 2Sz = 0 sector (dense)."""
    dim = 2 ** n
    H = np.zeros((dim, dim))
    for i in range(n - 1):
        for a, b, c in ((SZ, SZ, delta), (SP, SM, 0.5), (SM, SP, 0.5)):
            ops = [ID] * n
            ops[i], ops[i + 1] = a, b
            M = ops[0]
            for o in ops[1:]:
                M = np.kron(M, o)
            H += c * M
    idx = [s for s in range(dim) if bin(s).count("1") == n // 2]
    return float(np.linalg.eigvalsh(H[np.ix_(idx, idx)])[0])


# ── the single two-site H_eff of a canonical Heisenberg MPS (N = 16, chi = 64) ──

# Sector dimension profile over |2Sz| of the part left of a link: the centre
# link of N = 16 gets {4, 12, 32, 12, 4} on 2Sz = -4..4; every link keeps the
# charges of this profile that its sites allow, each at most the sector's
# Schmidt bound min(binom(b, .), binom(n - b, .)).
CENTER_PROFILE = {0: 32, 1: 22, 2: 12, 3: 8, 4: 4}


def profile_link(n: int, b: int) -> qn.U1Link:
    """Link after b of n sites: charges Q = 2Sz of the first b sites."""
    from math import comb
    m = min(b, n - b)
    charges, dims = [], []
    for q in range(-m, m + 1, 2):
        d = CENTER_PROFILE.get(abs(q), 0)
        bound = min(comb(b, (b + q) // 2), comb(n - b, (n - b - q) // 2))
        if d > 0 and bound > 0:
            charges.append(q)
            dims.append(min(d, bound))
    return qn.U1Link(charges, dims)


def _site_blocks(left: qn.U1Link, right: qn.U1Link, rng):
    """Seeded N(0, 1) blocks of A[(ql, s, qr) | (ml, mr)] on every allowed key."""
    out = {}
    for il, ql in enumerate(left.charges):
        for s in range(2):
            q = ql + qn.PHYS[s]
            if q in right.charges:
                ir = right.index(q)
                out[(il + 1, s + 1, ir + 1)] = rng.standard_normal((left.dims[il], right.dims[ir]))
    return out


def _bs_from_blocks(ctx, left, right, blocks):
    import sparsebackends_b200 as sb
    keys = sorted(blocks, key=lambda k: k[::-1])
    data = np.concatenate([blocks[k].reshape(-1, order="F") for k in keys])
    return sb.NewBlockSparseSorted((left.S, 2, right.S, left.D, right.D), 2, keys, None, data, ctx=ctx,
                                   block_dims=[blocks[k].shape for k in keys])


def _sector_qr(ctx, rows):
    """QR of one charge sector through the library's blocksparse_left_qr
    (ops_factorize.jl:8-43): ``rows`` = list of (s, matrix r_j x c) whose row
    blocks stack to M (sum r_j rows, c columns), given as A[(l, r) | (1)]
    (every row its own l, a unit tail).  Returns (the Q row blocks as (s,
    r_j x k), R (k x c)), M = Q R."""
    import sparsebackends_b200 as sb
    M = np.vstack([m for _, m in rows])
    nl, c = M.shape
    keys = [(l + 1, r + 1) for r in range(c) for l in range(nl)]
    data = np.array([M[l - 1, r - 1] for l, r in keys])
    A = sb.NewBlockSparseSorted((nl, c, 1), 1, keys, None, data, ctx=ctx)
    Q, R, lv, rv = sb.blocksparse_left_qr(A)
    Rm = R.to_numpy()
    k = Rm.shape[0]
    qb = Q.blocks_by_key()
    qfull = np.zeros((nl, k))
    for l in lv:
        qfull[l - 1] = np.asarray(qb[(l,)]).reshape(k)
    Rfull = np.zeros((k, c))
    Rfull[:, [r - 1 for r in rv]] = Rm
    out, off = [], 0
    for s, m in rows:
        out.append((s, qfull[off: off + m.shape[0]]))
        off += m.shape[0]
    return out, Rfull


def canonical_center_problem(ctx, n: int = 16, seed: int = 2026):
    """The two-site H_eff problem of a Heisenberg chain at its centre bond:
    links by ``profile_link`` (chi <= 64, centre {4, 12, 32, 12, 4}), seeded
    N(0, 1) site tensors, sites 1..n/2-1 left-canonicalised and sites
    n/2+2..n right-canonicalised by QR per charge sector (the library's
    blocksparse_left_qr), L and R built from the boundaries by make_L / make_R,
    and psi Gaussian on the flux-0 blocks of sites n/2, n/2+1, normalised.
    Returns (layout, psi, L, W, R)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    links = [profile_link(n, b) for b in range(n + 1)]
    sites = [_site_blocks(links[i], links[i + 1], rng) for i in range(n)]
    c = n // 2  # centre bond between sites c and c+1 (1-based)
    # left-canonicalise sites 1..c-1, absorbing R into the next site
    for i in range(c - 1):
        left, right = links[i], links[i + 1]
        newdims = list(right.dims)
        rs = {}
        for ir, q in enumerate(right.charges):
            rows = [(k[1], m) for k, m in sites[i].items() if k[2] == ir + 1]
            if not rows:
                continue
            qrows, R = _sector_qr(ctx, rows)
            for (s, qm), (k, _) in zip(qrows, [(k, m) for k, m in sites[i].items() if k[2] == ir + 1]):
                sites[i][k] = qm
            rs[ir] = R
            newdims[ir] = R.shape[0]
        for k in list(sites[i + 1]):
            if k[0] - 1 in rs:
                sites[i + 1][k] = rs[k[0] - 1] @ sites[i + 1][k]
        links[i + 1] = qn.U1Link(list(right.charges), newdims)
    # right-canonicalise sites n..c+2, absorbing R^T into the previous site
    for i in range(n - 1, c, -1):
        left = links[i]
        newdims = list(left.dims)
        rs = {}
        for il, q in enumerate(left.charges):
            items = [(k, m) for k, m in sites[i].items() if k[0] == il + 1]
            if not items:
                continue
            # transposed: rows (mr, s), columns ml
            qrows, R = _sector_qr(ctx, [(k[1], m.T) for k, m in items])
            for (s, qm), (k, _) in zip(qrows, items):
                sites[i][k] = qm.T
            rs[il] = R
            newdims[il] = R.shape[0]
        for k in list(sites[i - 1]):
            if k[2] - 1 in rs:
                sites[i - 1][k] = sites[i - 1][k] @ rs[k[2] - 1].T
        links[i] = qn.U1Link(list(left.charges), newdims)
    W = mpo_tensor(ctx, 1.0)
    L, R = boundary_envs(ctx)
    for i in range(c - 1):
        L = qn.make_L(L, _bs_from_blocks(ctx, links[i], links[i + 1], sites[i]), W)
    for i in range(n - 1, c, -1):
        R = qn.make_R(R, _bs_from_blocks(ctx, links[i], links[i + 1], sites[i]), W)
    lay = qn.HeffLayout(links[c - 1], links[c + 1], MPO_LINK)
    import sparsebackends_b200 as sb
    keys, data, exts = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    data = data / np.linalg.norm(data)
    psi = sb.NewBlockSparseSorted(lay.dims["psi"], lay.n2["psi"], keys, None, data, ctx=ctx, block_dims=exts)
    return lay, psi, L, W, R
