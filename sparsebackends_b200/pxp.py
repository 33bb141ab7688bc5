"""PXP chain (Rydberg blockade): H = sum_i P_{i-1} X_i P_{i+1}, P = |0><0|,
open boundaries, no conserved charge.

The MPO is the lower-triangular bond-4 one (channels 1 = done, 2 = P X placed,
3 = P placed, 4 = nothing placed yet; the left boundary selects channel 4, the
right boundary channel 1), 8 nonzero entries of 64 in 5 of the 16 (wl, wr)
blocks, stored as a COOTensor W[s', s, wl, wr] (the MPO storage of
test_pxp_sparse.jl:377-411, src/coo/storage.jl:1-6).

Links carry no charge, so each maps onto the reference format as (sector
prefix axis of extent 1, dense tail axis): an MPS site tensor is block-sparse
(ql, s, qr | l, r) with one block per physical value, an environment
(q', w, q | m', m) with one block per MPO channel.  The MPO enters every
contraction the way contract_prefix! (contract_coo_bs.jl:51-124) takes it: the
physical index and the MPO link it meets are fused into one prefix label on
both sides (fuse_axes_coo, coo/conversions.jl:174-222; fuse_two_axes!,
blocksparse/conversions.jl:228-262), and the single fused label is reduced by
scaled block adds.  The dense contractions (environment times state) are
contract_shared! calls (contract_bs_bs.jl:572-730), on the tensor cores in a
context whose precision is "tf32x3".

Every step table below is chosen so that no dense tail is permuted: each
contract_shared! operand already has its tail in the join order the kernel
needs (kept then reduced for the left operand, reduced then kept for the
right one), and each fused pair is adjacent with the reduced label last.
"""
from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np

D = 2  # physical dimension
W = 4  # MPO bond dimension

# (wl, wr, operator), 0-based channels of the bond-4 MPO
CHANNELS = ((0, 0, "I"), (1, 0, "P"), (2, 1, "X"), (3, 2, "P"), (3, 3, "I"))
OPS = {"I": np.eye(D), "P": np.array([[1.0, 0.0], [0.0, 0.0]]), "X": np.array([[0.0, 1.0], [1.0, 0.0]])}
LEFT_CHANNEL, RIGHT_CHANNEL = 4, 1  # 1-based boundary channels

# Labels of the operands (prefix | tail).
LABELS = {
    "psi": ("ql", "s1", "s2", "qr", "l", "r"),
    "A": ("ql", "s", "qr", "l", "r"),          # one-site MPS tensor
    "Abar": ("qlp", "sp", "qrp", "lp", "rp"),  # its conjugate (real: the same tensor)
    "L": ("qlp", "wl", "ql", "lp", "l"),
    "R": ("qrp", "wr", "qr", "r", "rp"),
    # W with the physical index and one MPO link fused, the fused label last
    # (the reduced label of contract_prefix!, so no per-call permute and sort)
    "Wf": ("sp", "wr", "x"),                   # x = (wl-1)*D + s
    "Wrf": ("sp", "wl", "x"),                  # x = (wr-1)*D + s
    "W1f": ("s1p", "wm", "x1"),
    "W2f": ("s2p", "wr", "x2"),
}

# The aliased form: W as AliasedBlockSparse (prefix (wl, wr) | tail (s', s)),
# one template per distinct one-site operator (I, P, X), and dense psi and
# environments.  Every step is a contract_shared! / contract! of the aliased
# backend (contract_aliased_shared.jl:103-302 Aliased x Dense,
# :325-523 Aliased x Aliased; contract_aliased.jl:244-365): the MPO products
# are formed once per (template, template) or (template, slice) pair and
# shared by every key that uses them; keys that collect several distinct
# products are accumulated into a block of their own.
ALIASED_LABELS = {
    "psi_d": ("l", "s1", "s2", "r"),
    "Ld": ("lp", "wl", "l"),
    "Rd": ("rp", "wr", "r"),
    "W1a": ("wl", "wm", "s1p", "s1"),
    "W2a": ("wm", "wr", "s2p", "s2"),
}
ALIASED_HEFF_STEPS = (
    ("contract", "X1", ("wl", "wm", "s1p", "l", "s2", "r"), 4, "W1a", "psi_d"),
    ("contract", "X2", ("wl", "wr", "s1p", "l", "r", "s2p"), 4, "W2a", "X1"),
    ("contract", "X3", ("wr", "lp", "s1p", "r", "s2p"), 4, "X2", "Ld"),
    ("contract", "X4", ("lp", "s1p", "s2p", "rp"), 4, "X3", "Rd"),  # no prefix: one key (), H_eff . psi
)

# ("contract", result, result labels, result tail count, left, right) or
# ("fuse", result, operand, ax1, ax2, fused label); ax1 is the fast index.
ENV_L_STEPS = (
    ("contract", "E1", ("qlp", "qr", "s", "wl", "r", "lp"), 2, "L", "A"),
    ("fuse", "E1f", "E1", 3, 4, "x"),
    ("contract", "E2", ("qlp", "sp", "wr", "qr", "r", "lp"), 2, "Wf", "E1f"),
    ("contract", "out", ("qrp", "wr", "qr", "rp", "r"), 2, "E2", "Abar"),
)
ENV_R_STEPS = (
    ("contract", "F1", ("ql", "qrp", "s", "wr", "rp", "l"), 2, "A", "R"),
    ("fuse", "F1f", "F1", 3, 4, "x"),
    ("contract", "F2", ("ql", "sp", "wl", "qrp", "rp", "l"), 2, "Wrf", "F1f"),
    ("contract", "out", ("qlp", "wl", "ql", "l", "lp"), 2, "Abar", "F2"),
)
HEFF_STEPS = (
    ("contract", "T1", ("qlp", "s2", "qr", "s1", "wl", "lp", "r"), 2, "L", "psi"),
    ("fuse", "T1f", "T1", 4, 5, "x1"),
    ("contract", "T2", ("qlp", "s1p", "qr", "s2", "wm", "lp", "r"), 2, "W1f", "T1f"),
    ("fuse", "T2f", "T2", 4, 5, "x2"),
    ("contract", "T3", ("qlp", "s1p", "s2p", "wr", "qr", "lp", "r"), 2, "W2f", "T2f"),
    ("contract", "T4", ("qlp", "s1p", "s2p", "qrp", "lp", "rp"), 2, "T3", "R"),
)


def run_steps(steps, tensors: Dict, labels: Dict, contract, fuse) -> Dict:
    """Run a step table.  ``contract(labelsC, n2C, A, labelsA, B, labelsB)``
    returns a new result; ``fuse(A, ax1, ax2)`` returns A with the two axes
    fused (1-based).  ``tensors`` and ``labels`` gain the results."""
    for st in steps:
        if st[0] == "contract":
            _, c, lc, n2, a, b = st
            tensors[c] = contract(list(lc), n2, tensors[a], list(labels[a]), tensors[b], list(labels[b]))
            labels[c] = tuple(lc)
        else:
            _, c, a, ax1, ax2, name = st
            tensors[c] = fuse(tensors[a], ax1, ax2)
            lab = list(labels[a])
            lab[ax1 - 1] = name
            del lab[ax2 - 1]
            labels[c] = tuple(lab)
    return tensors


def mpo_dense() -> np.ndarray:
    """W[s', s, wl, wr] of one site."""
    Wd = np.zeros((D, D, W, W))
    for wl, wr, op in CHANNELS:
        Wd[:, :, wl, wr] = OPS[op]
    return Wd


def mpo_entries():
    """1-based keys (s', s, wl, wr) and values of W's nonzero entries,
    column-major sorted (the order sort_coo! leaves)."""
    Wd = mpo_dense()
    idx = np.argwhere(Wd != 0.0)
    keys = sorted((tuple(int(i) + 1 for i in k) for k in idx), key=lambda k: tuple(reversed(k)))
    return keys, [float(Wd[tuple(x - 1 for x in k)]) for k in keys]


def mpo_aliased():
    """(dims, templates, keys, alias_ids, scalars) of W as an aliased tensor
    (wl, wr | s', s): templates I, P, X (column-major 2x2), keys sorted
    column-major, every scalar 1."""
    names = ("I", "P", "X")
    keys = sorted(((wl + 1, wr + 1) for wl, wr, _ in CHANNELS), key=lambda k: (k[1], k[0]))
    op = {(wl + 1, wr + 1): o for wl, wr, o in CHANNELS}
    templates = np.concatenate([OPS[m].reshape(-1, order="F") for m in names])
    return (W, W, D, D), templates, keys, [names.index(op[k]) + 1 for k in keys], [1.0] * len(keys)


def env_dense(keys: Sequence, blocks: Dict, dims: Sequence[int], right: bool) -> np.ndarray:
    """Dense E[m', w, m] from environment blocks (left layout (q', w, q | m',
    m); right layout (q', w, q | m, m'))."""
    m1, m2 = dims[3], dims[4]
    out = np.zeros((m2, dims[1], m1) if right else (m1, dims[1], m2))
    for k in keys:
        b = np.asarray(blocks[k]).reshape(m1, m2, order="F")
        out[:, k[1] - 1, :] = b.T if right else b
    return out


def bond_dims(n: int, chi: int) -> List[int]:
    """D_0..D_n: the bond after site k is min(d^k, d^(n-k), chi)."""
    return [min(D ** k, D ** (n - k), chi) for k in range(n + 1)]


def random_mps(n: int, chi: int, seed: int):
    """A random MPS with the orthogonality centre on the two middle sites.

    Returns (sites, psi, c): ``sites[k]`` (k = 0..n-1) the host array
    A[l, s, r] of site k+1 for every site but c, c+1 (1-based), with N(0,1)
    draws made isometric by QR: left-canonical left of the centre
    (sum_s A_s^T A_s = 1), right-canonical right of it (sum_s A_s A_s^T = 1);
    ``psi`` the two-site centre tensor psi[l, s1, s2, r], N(0,1), unit norm."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dims = bond_dims(n, chi)
    c = n // 2  # 1-based left centre site
    sites: List = [None] * n
    for k in range(1, c):
        dl, dr = dims[k - 1], dims[k]
        q, _ = np.linalg.qr(rng.standard_normal((dl * D, dr)))
        sites[k - 1] = q.reshape(dl, D, dr, order="F")
    for k in range(n, c + 1, -1):
        dl, dr = dims[k - 1], dims[k]
        q, _ = np.linalg.qr(rng.standard_normal((D * dr, dl)))
        sites[k - 1] = np.ascontiguousarray(q.T).reshape(dl, D, dr, order="F")
    psi = rng.standard_normal((dims[c - 1], D, D, dims[c + 1]))
    psi /= np.linalg.norm(psi)
    return sites, psi, c


def site_blocks(A: np.ndarray):
    """(dims, keys, data) of a site tensor A[l, s, r] as block-sparse
    (ql, s, qr | l, r): one block per physical value."""
    dl, d, dr = A.shape
    keys = [(1, s + 1, 1) for s in range(d)]
    data = np.concatenate([A[:, s, :].reshape(-1, order="F") for s in range(d)])
    return (1, d, 1, dl, dr), keys, data


def psi_blocks(psi: np.ndarray):
    """(dims, keys, data) of psi[l, s1, s2, r] as block-sparse
    (ql, s1, s2, qr | l, r), keys column-major sorted."""
    dl, d1, d2, dr = psi.shape
    keys, parts = [], []
    for s2 in range(d2):
        for s1 in range(d1):
            keys.append((1, s1 + 1, s2 + 1, 1))
            parts.append(psi[:, s1, s2, :].reshape(-1, order="F"))
    return (1, d1, d2, 1, dl, dr), keys, np.concatenate(parts)


def boundary_blocks(channel: int):
    """(dims, keys, data) of a boundary environment: one 1x1 block at the
    boundary channel."""
    return (1, W, 1, 1, 1), [(1, channel, 1)], np.ones(1)


def psi_from_blocks(keys: Sequence, data: np.ndarray, dims: Sequence[int]) -> np.ndarray:
    """Dense psi[l, s1, s2, r] from (ql, s1, s2, qr | l, r) blocks."""
    dl, dr = dims[4], dims[5]
    out = np.zeros((dl, dims[1], dims[2], dr))
    blk = dl * dr
    for i, k in enumerate(keys):
        out[:, k[1] - 1, k[2] - 1, :] = data[i * blk:(i + 1) * blk].reshape(dl, dr, order="F")
    return out


class PxpProblem:
    """The two-site centre problem of a random PXP MPS on the device.

    ``n`` sites, bond dimension up to ``chi``; the environments L (sites
    1..c-1) and R (sites c+2..n) are built by ``make_L`` / ``make_R`` from the
    boundaries, three contractions and one fusion per site, all on the device."""

    def __init__(self, n: int = 64, chi: int = 256, seed: int = 64, ctx=None):
        import sparsebackends_b200 as sb
        self.sb = sb
        self.ctx = ctx or sb.default_context()
        self.n, self.chi, self.seed = n, chi, seed
        self.sites, self.psi_host, self.c = random_mps(n, chi, seed)
        keys, vals = mpo_entries()
        self.W = sb.COOTensor((D, D, W, W), keys, vals, ctx=self.ctx)
        self.Wf = sb.fuse_axes(sb.permutedims(self.W, [1, 4, 2, 3]), 3, 4)   # (s', wr, x)
        self.Wrf = sb.fuse_axes(sb.permutedims(self.W, [1, 3, 2, 4]), 3, 4)  # (s', wl, x)
        self.Ws = sb.sort_(sb.permutedims(self.W, [1, 3, 4, 2]))             # (s', wl, wr, s)
        L = self._bs(*boundary_blocks(LEFT_CHANNEL))
        for k in range(1, self.c):
            L = self.make_L(L, self._bs(*site_blocks(self.sites[k - 1])))
        R = self._bs(*boundary_blocks(RIGHT_CHANNEL))
        for k in range(n, self.c + 1, -1):
            R = self.make_R(R, self._bs(*site_blocks(self.sites[k - 1])))
        self.L, self.R = L, R
        self.psi = self._bs(*psi_blocks(self.psi_host))

    def _bs(self, dims, keys, data):
        return self.sb.NewBlockSparseSorted(dims, 2, keys, data=data, ctx=self.ctx)

    def _contract(self, lc, n2, A, la, B, lb):
        ext = dict(zip(la, A.dims))
        ext.update(zip(lb, B.dims))
        C = self.sb.NewBlockSparseSorted.empty(tuple(ext[x] for x in lc), n2, ctx=self.ctx)
        return self.sb.contract_(C, lc, A, la, B, lb)

    def _run(self, steps, tensors):
        return run_steps(steps, tensors, dict(LABELS), self._contract, self.sb.fuse_axes)

    def make_L(self, L, A):
        """L' = L . A . W . Abar (ITensorMPS makeL!)."""
        return self._run(ENV_L_STEPS, {"L": L, "A": A, "Abar": A, "Wf": self.Wf})["out"]

    def make_R(self, R, B):
        """R' = R . B . W . Bbar (ITensorMPS makeR!)."""
        return self._run(ENV_R_STEPS, {"R": R, "A": B, "Abar": B, "Wrf": self.Wrf})["out"]

    def apply(self, psi):
        """H_eff . psi in psi's layout: psi.L, .W1, .W2, .R (product(::ProjMPO, v)
        order), four contractions and two fusions."""
        return self._run(HEFF_STEPS, {"psi": psi, "L": self.L, "R": self.R, "W1f": self.Wf,
                                      "W2f": self.Wf})["T4"]

    def aliased_operands(self):
        """The aliased form's operands on the device: W as an aliased tensor
        and dense L, R (converted from the block environments once)."""
        sb = self.sb
        dims, tm, keys, aids, sc = mpo_aliased()
        Wa = sb.AliasedBlockSparse(dims, 2, tm, keys, aids, sc, ctx=self.ctx)
        Ld = sb.DenseTensor(env_dense(self.L.keys, self.L.blocks_by_key(), self.L.dims, right=False), ctx=self.ctx)
        Rd = sb.DenseTensor(env_dense(self.R.keys, self.R.blocks_by_key(), self.R.dims, right=True), ctx=self.ctx)
        return {"W1a": Wa, "W2a": Wa, "Ld": Ld, "Rd": Rd}

    def apply_aliased(self, psi_d, ops):
        """H_eff . psi with the MPO in aliased storage: ``psi_d`` a dense
        DenseTensor (l, s1, s2, r), ``ops`` from ``aliased_operands``.  Returns
        an aliased tensor with one key () whose logical block is H_eff . psi in
        psi's layout."""
        sb = self.sb

        def contract(lc, n2, A, la, B, lb):
            ext = dict(zip(la, A.dims))
            ext.update(zip(lb, B.dims))
            C = sb.AliasedBlockSparse.empty(tuple(ext[x] for x in lc), n2, ctx=self.ctx)
            return sb.contract_(C, lc, A, la, B, lb)

        return run_steps(ALIASED_HEFF_STEPS, {"psi_d": psi_d, **ops}, dict(ALIASED_LABELS), contract, None)["X4"]

    def capture(self, psi):
        """Run the matvec once, then capture it as one CUDA graph bound to
        ``psi``'s payload.  Returns (graph, out): ``graph.launch()`` recomputes
        ``out`` from the current values of ``psi``; the intermediates are
        allocated at capture and live as long as the graph."""
        self.apply(psi)
        box = {}
        graph = self.ctx.capture(lambda: box.setdefault("out", self.apply(psi)), keep=[psi, self.L, self.R, self.Wf])
        graph.hold(box["out"])
        return graph, box["out"]

    def apply_mpo(self, A):
        """MPO x MPS on one site tensor (ql, s, qr | l, r): C(s', wl, wr, ql, qr |
        l, r) = sum_s W(s', s, wl, wr) A(ql, s, qr | l, r), COO x block-sparse
        (contract_prefix!; W is kept with s last, A's s moves last in its prefix)."""
        dims = (D, W, W, 1, 1) + tuple(A.dims[3:])
        C = self.sb.NewBlockSparseSorted.empty(dims, 2, ctx=self.ctx)
        return self.sb.contract_(C, ["sp", "wl", "wr", "ql", "qr", "l", "r"], self.Ws, ["sp", "wl", "wr", "s"],
                                 A, ["ql", "s", "qr", "l", "r"])
