"""The J1-J2 Heisenberg model on a cylinder as a U(1) MPO for ``dmrg.DMRG``.

H = sum_<ij> J_ij (Sz_i Sz_j + (S+_i S-_j + S-_i S+_j) / 2) on an lx x ly
cylinder (open along x, periodic along y), J1 on nearest and J2 on
next-nearest (diagonal) neighbours, sites in snake order (column x runs up for
even x, down for odd x).

The MPO is the finite-automaton one (ITensors' OpSum construction before its
SVD compression).  At the bond after site b, the channels are:
"start" (nothing placed), "done" (a term completed), and for every site i <= b
that still has a partner j > b, three channels "S+ placed at i", "S- placed at
i", "Sz placed at i".  A channel carries the charge of its operator (2Sz
units: +2, -2, 0), so the link is graded like the XXZ chain's, with the
coupling applied where a term closes.  Every bond's channels are laid out in
one padded link (the largest count of each charge over the bonds), so all
sites share one MPO link in the H_eff layout; unused channels hold no blocks'
entries.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

from . import qn
from .dmrg import ID, SM, SP, SZ

START, DONE = 1, 2  # 1-based positions in the charge-0 sector


def snake_index(x: int, y: int, ly: int) -> int:
    return x * ly + (y if x % 2 == 0 else ly - 1 - y)


def cylinder_couplings(lx: int, ly: int, j1: float = 1.0, j2: float = 0.5) -> Dict[Tuple[int, int], float]:
    """{(i, j): J_ij} over 0-based snake-ordered sites, i < j.  Each nearest-
    and next-nearest-neighbour pair counts once, also on a narrow cylinder
    where the periodic wrap reaches the same site twice."""
    nn, nnn = set(), set()

    def pair(a, b):
        return (min(a, b), max(a, b))

    for x in range(lx):
        for y in range(ly):
            a = snake_index(x, y, ly)
            if ly > 1:
                nn.add(pair(a, snake_index(x, (y + 1) % ly, ly)))
            if x + 1 < lx:
                nn.add(pair(a, snake_index(x + 1, y, ly)))
                if ly > 1:
                    nnn.add(pair(a, snake_index(x + 1, (y + 1) % ly, ly)))
                    nnn.add(pair(a, snake_index(x + 1, (y - 1) % ly, ly)))
    out: Dict[Tuple[int, int], float] = {}
    for p in nn:
        if p[0] != p[1] and j1 != 0.0:
            out[p] = out.get(p, 0.0) + j1
    for p in nnn:
        if p[0] != p[1] and j2 != 0.0:
            out[p] = out.get(p, 0.0) + j2
    return dict(sorted(out.items()))


class J1J2Cylinder:
    """The MPO of ``cylinder_couplings(lx, ly, j1, j2)``: ``link`` (the padded
    U(1) MPO link), ``site_blocks(k)`` (host blocks of site k's W), device
    tensors via ``tensors(ctx)`` and boundary environments via
    ``boundary_envs(ctx)``."""

    def __init__(self, lx: int = 6, ly: int = 6, j1: float = 1.0, j2: float = 0.5):
        self.lx, self.ly, self.n = lx, ly, lx * ly
        self.J = cylinder_couplings(lx, ly, j1, j2)
        last = {}
        for (i, j) in self.J:
            last[i] = max(last.get(i, -1), j)
        self.last = last  # last partner of each site
        n = self.n
        # open[b]: sites i <= b with a partner beyond b, for the bond after site b (b = -1 .. n-1)
        self.open = {b: [i for i in range(b + 1) if last.get(i, -1) > b] for b in range(-1, n)}
        k = max(len(v) for v in self.open.values())
        self.link = qn.mpo_link({-2: max(k, 1), 0: 2 + k, 2: max(k, 1)})

    def _pos(self, b: int, ch) -> Tuple[int, int]:
        """(1-based sector, 1-based index in the sector) of a channel at the
        bond after site b: "start", "done" or (site, "+" | "-" | "z")."""
        w = self.link
        if ch == "start":
            return w.index(0) + 1, START
        if ch == "done":
            return w.index(0) + 1, DONE
        i, op = ch
        r = self.open[b].index(i)
        if op == "z":
            return w.index(0) + 1, 3 + r
        return w.index(2 if op == "+" else -2) + 1, 1 + r

    def terms(self, k: int):
        """(left channel, right channel, operator) of site k's W."""
        out = [("start", "start", ID), ("done", "done", ID)]
        if self.last.get(k, -1) > k:
            out += [("start", (k, "+"), SP), ("start", (k, "-"), SM), ("start", (k, "z"), SZ)]
        for i in self.open[k - 1]:
            if self.last[i] > k:
                for op in "+-z":
                    out.append(((i, op), (i, op), ID))
            j = self.J.get((i, k), 0.0)
            if j != 0.0:
                out += [((i, "+"), "done", 0.5 * j * SM), ((i, "-"), "done", 0.5 * j * SP), ((i, "z"), "done", j * SZ)]
        return out

    def site_blocks(self, k: int):
        """Host blocks of W_k[(qwl, s', s, qwr) | (mwl, mwr)] at the padded
        sector extents."""
        w = self.link
        blocks = {}
        for cl, cr, op in self.terms(k):
            (ql, ml), (qr, mr) = self._pos(k - 1, cl), self._pos(k, cr)
            for sp in range(2):
                for s in range(2):
                    if op[sp, s] == 0.0:
                        continue
                    key = (ql, sp + 1, s + 1, qr)
                    blk = blocks.setdefault(key, np.zeros((w.dims[ql - 1], w.dims[qr - 1])))
                    blk[ml - 1, mr - 1] += op[sp, s]
        return blocks

    def tensors(self, ctx) -> List:
        import sparsebackends_b200 as sb
        w = self.link
        out = []
        for k in range(self.n):
            blocks = self.site_blocks(k)
            keys = sorted(blocks, key=lambda q: q[::-1])
            data = np.concatenate([blocks[q].reshape(-1, order="F") for q in keys])
            out.append(sb.NewBlockSparseSorted((w.S, 2, 2, w.S, w.D, w.D), 2, keys, None, data, ctx=ctx,
                                               block_dims=[blocks[q].shape for q in keys]))
        return out

    def boundary_envs(self, ctx):
        """L0 on "start", R0 on "done" (charge-0 sector, bond sectors of dimension 1)."""
        import sparsebackends_b200 as sb
        w = self.link
        q0 = w.index(0) + 1
        d0 = w.dims[q0 - 1]
        l0, r0 = np.zeros(d0), np.zeros(d0)
        l0[START - 1] = 1.0
        r0[DONE - 1] = 1.0
        dims = (1, w.S, 1, 1, w.D, 1)
        L = sb.NewBlockSparseSorted(dims, 3, [(1, q0, 1)], None, l0, ctx=ctx, block_dims=[(1, d0, 1)])
        R = sb.NewBlockSparseSorted(dims, 3, [(1, q0, 1)], None, r0, ctx=ctx, block_dims=[(1, d0, 1)])
        return L, R

    def dense_mpo(self, k: int) -> np.ndarray:
        """W_k as a dense array [wl, wr, s', s] over the flat padded channel
        index (sectors in link order)."""
        w = self.link
        off = np.concatenate([[0], np.cumsum(w.dims)])
        tot = int(off[-1])
        out = np.zeros((tot, tot, 2, 2))
        for (ql, sp, s, qr), blk in self.site_blocks(k).items():
            out[off[ql - 1]:off[ql - 1] + blk.shape[0], off[qr - 1]:off[qr - 1] + blk.shape[1], sp - 1, s - 1] += blk
        return out

    def boundary_vectors(self) -> Tuple[np.ndarray, np.ndarray]:
        w = self.link
        off = np.concatenate([[0], np.cumsum(w.dims)])
        q0 = w.index(0)
        l, r = np.zeros(int(off[-1])), np.zeros(int(off[-1]))
        l[off[q0] + START - 1] = 1.0
        r[off[q0] + DONE - 1] = 1.0
        return l, r


def dense_hamiltonian(n: int, J: Dict[Tuple[int, int], float]) -> np.ndarray:
    """H over n spins (site 0 the most significant factor of the Kronecker
    products), from the couplings directly."""
    dim = 2 ** n
    H = np.zeros((dim, dim))
    for (i, j), c in J.items():
        for a, b, f in ((SZ, SZ, 1.0), (SP, SM, 0.5), (SM, SP, 0.5)):
            ops = [ID] * n
            ops[i], ops[j] = a, b
            M = ops[0]
            for o in ops[1:]:
                M = np.kron(M, o)
            H += c * f * M
    return H


def exact_ground_energy(n: int, J: Dict[Tuple[int, int], float]) -> float:
    """Lowest eigenvalue in the total 2Sz = 0 sector (dense, small n)."""
    H = dense_hamiltonian(n, J)
    idx = [s for s in range(2 ** n) if bin(s).count("1") == n // 2]
    return float(np.linalg.eigvalsh(H[np.ix_(idx, idx)])[0])
