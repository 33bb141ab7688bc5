"""U(1) sectors on the reference's block-sparse format, and the two-site H_eff apply.

The reference stores every tensor as ``NewBlockSparseSorted`` (prefix-sparse,
tail-dense, uniform block size).  A U(1)-graded link becomes two axes:

* a prefix axis ``q`` over its charge sectors (keys = allowed sector tuples);
* a tail axis ``m`` over the states inside a sector, zero-padded to the
  largest sector dimension ``D``.

Blocks exist only for charge-conserving sector tuples.  The MPO link is graded
the same way (its channels grouped by the charge they carry: -2, 0, +2), which
keeps the H_eff chain at the MPS' block sparsity.

``HeffChain`` applies the two-site effective Hamiltonian in the order of
ITensorMPS ``product(::ProjMPO, v)`` (ψ·L, ·W₁, ·W₂, ·R), as four
``contract!`` calls (``src/tensoralgebra/contract_bs_bs.jl:572-730``).  Label
orders are chosen so that each call's operand permutations are key reorders
only: every dense tail already sits in the [kept..., reduced...] order the
kernel wants.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np


@dataclass
class U1Link:
    """Charge sectors of one link: ``charges[i]`` with ``dims[i]`` states."""

    charges: List[int]
    dims: List[int]

    @property
    def S(self) -> int:
        return len(self.charges)

    @property
    def D(self) -> int:
        return max(self.dims)

    @property
    def total(self) -> int:
        return int(sum(self.dims))

    def index(self, q: int) -> int:
        return self.charges.index(q)


PHYS = [+1, -1]  # 2Sz of the spin-1/2 states s = 1, 2


def gaussian_sectors(chi: int, charges: Sequence[int], width: float, min_dim: int = 1) -> U1Link:
    """Sector dims ∝ exp(-(q/2)²/(2 width²)) summing to ``chi`` (a DMRG-like profile)."""
    w = np.exp(-((np.asarray(charges) / 2.0) ** 2) / (2 * width ** 2))
    raw = w / w.sum() * chi
    dims = np.maximum(min_dim, np.floor(raw)).astype(int)
    # distribute the remainder to the largest fractional parts
    rem = chi - int(dims.sum())
    order = np.argsort(-(raw - np.floor(raw)))
    i = 0
    while rem > 0:
        dims[order[i % len(dims)]] += 1
        rem -= 1
        i += 1
    while rem < 0:
        j = int(np.argmax(dims))
        dims[j] -= 1
        rem += 1
    return U1Link(list(charges), [int(d) for d in dims])


def mpo_link(channels_per_charge: Dict[int, int]) -> U1Link:
    """MPO link graded by channel charge, e.g. {-2: k, 0: 2+k, 2: k}."""
    qs = sorted(channels_per_charge)
    return U1Link(qs, [channels_per_charge[q] for q in qs])


@dataclass
class HeffLayout:
    """Dims, tail counts, labels and charge-allowed keys of every tensor in the chain."""

    left: U1Link
    right: U1Link
    mpo: U1Link
    d: int = 2
    labels: Dict[str, List[str]] = field(default_factory=dict)
    dims: Dict[str, Tuple[int, ...]] = field(default_factory=dict)
    n2: Dict[str, int] = field(default_factory=dict)
    keys: Dict[str, List[Tuple[int, ...]]] = field(default_factory=dict)

    def __post_init__(self):
        l, r, w, d = self.left, self.right, self.mpo, self.d
        S_l, S_r, S_w, D_l, D_r, D_w = l.S, r.S, w.S, l.D, r.D, w.D
        ext = {"ql": S_l, "qlp": S_l, "qr": S_r, "qrp": S_r, "qwl": S_w, "qwm": S_w, "qwr": S_w,
               "s1": d, "s2": d, "s1p": d, "s2p": d,
               "ml": D_l, "mlp": D_l, "mr": D_r, "mrp": D_r, "mwl": D_w, "mwm": D_w, "mwr": D_w}
        lab = {
            "psi": ["ql", "s1", "s2", "qr", "ml", "mr"],
            "L": ["qlp", "qwl", "ql", "mlp", "mwl", "ml"],
            "W1": ["qwl", "s1p", "s1", "qwm", "mwl", "mwm"],
            "W2": ["qwm", "s2p", "s2", "qwr", "mwm", "mwr"],
            "R": ["qrp", "qwr", "qr", "mrp", "mwr", "mr"],
            # intermediates: orders chosen so that no dense tail needs a permute
            "T1": ["qlp", "s2", "qr", "qwl", "s1", "mr", "mlp", "mwl"],
            "T2": ["qlp", "qr", "s1p", "qwm", "s2", "mr", "mlp", "mwm"],
            "T3": ["qlp", "s1p", "s2p", "qwr", "qr", "mwr", "mr", "mlp"],
            "T4": ["qlp", "s1p", "s2p", "qrp", "mlp", "mrp"],
            # two-site MPO W1·W2 (the alternative association of the chain)
            "W12": ["qwl", "s1p", "s1", "s2p", "s2", "qwr", "mwl", "mwr"],
            # one-site MPS tensor (environment updates)
            "A": ["ql", "s1", "qr", "ml", "mr"],
        }
        n2 = {"psi": 2, "L": 3, "W1": 2, "W2": 2, "R": 3, "T1": 3, "T2": 3, "T3": 3, "T4": 2, "A": 2, "W12": 2}
        self.labels = lab
        self.n2 = n2
        self.dims = {k: tuple(ext[x] for x in v) for k, v in lab.items()}
        self.ext = ext
        self.keys = {
            "psi": self._psi_keys(),
            "L": self._env_keys(l),
            "W1": self._mpo_keys(),
            "W2": self._mpo_keys(),
            "R": self._env_keys(r),
            "A": self._site_keys(),
        }

    # ψ(ql, s1, s2, qr): Q(ql) + σ1 + σ2 = Q(qr)
    def _psi_keys(self):
        out = []
        for ql, s1, s2, qr in itertools.product(range(self.left.S), range(self.d), range(self.d), range(self.right.S)):
            if self.left.charges[ql] + PHYS[s1] + PHYS[s2] == self.right.charges[qr]:
                out.append((ql + 1, s1 + 1, s2 + 1, qr + 1))
        return out

    # A(ql, s, qr): Q(ql) + σ = Q(qr)
    def _site_keys(self):
        out = []
        for ql, s, qr in itertools.product(range(self.left.S), range(self.d), range(self.right.S)):
            if self.left.charges[ql] + PHYS[s] == self.right.charges[qr]:
                out.append((ql + 1, s + 1, qr + 1))
        return out

    # L(q', qw, q) / R(q', qw, q): Q(q') - Q(q) = c(qw)
    def _env_keys(self, link: U1Link):
        out = []
        for qp, qw, q in itertools.product(range(link.S), range(self.mpo.S), range(link.S)):
            if link.charges[qp] - link.charges[q] == self.mpo.charges[qw]:
                out.append((qp + 1, qw + 1, q + 1))
        return out

    # W(qwl, s', s, qwr): c(qwr) = c(qwl) + σ(s') - σ(s)
    def _mpo_keys(self):
        out = []
        w = self.mpo
        for a, sp, s, b in itertools.product(range(w.S), range(self.d), range(self.d), range(w.S)):
            if w.charges[b] == w.charges[a] + PHYS[sp] - PHYS[s]:
                out.append((a + 1, sp + 1, s + 1, b + 1))
        return out

    def valid_extent(self, name: str, key: Tuple[int, ...]) -> Tuple[int, ...]:
        """Unpadded extents of a block's tail axes (the rest is zero padding)."""
        lab = self.labels[name]
        P = len(lab) - self.n2[name]
        kv = {l: key[i] for i, l in enumerate(lab[:P])}
        grade = {"ml": ("ql", self.left), "mlp": ("qlp", self.left), "mr": ("qr", self.right),
                 "mrp": ("qrp", self.right), "mwl": ("qwl", self.mpo), "mwm": ("qwm", self.mpo),
                 "mwr": ("qwr", self.mpo)}
        out = []
        for t in lab[P:]:
            q, link = grade[t]
            out.append(link.dims[kv[q] - 1] if q in kv else link.D)
        return tuple(out)


def random_block_tensor(layout: HeffLayout, name: str, rng: np.random.Generator, scale: float = 1.0,
                        ragged: bool = False):
    """Gaussian entries inside each block's sector extents, zero padding outside.

    Returns (keys, data) in the reference layout (keys sorted column-major,
    blocks packed in that order).  With ``ragged=True`` returns
    (keys, data, block_dims): the same entries stored unpadded, block by block."""
    lab = layout.labels[name]
    dims = layout.dims[name]
    n2 = layout.n2[name]
    P = len(dims) - n2
    tail = dims[P:]
    blk = int(np.prod(tail))
    keys = layout.keys[name]
    pd = dims[:P]

    def lin(k):
        idx, st = 0, 1
        for a in range(P):
            idx += (k[a] - 1) * st
            st *= pd[a]
        return idx

    keys = sorted(keys, key=lin)
    if ragged:
        exts = [layout.valid_extent(name, k) for k in keys]
        parts = [(rng.standard_normal(e) * scale).reshape(-1, order="F") for e in exts]
        return keys, (np.concatenate(parts) if parts else np.zeros(0)), exts
    data = np.zeros(len(keys) * blk)
    for i, k in enumerate(keys):
        ext = layout.valid_extent(name, k)
        blkarr = np.zeros(tail)
        blkarr[tuple(slice(0, e) for e in ext)] = rng.standard_normal(ext) * scale
        data[i * blk:(i + 1) * blk] = blkarr.reshape(-1, order="F")
    return keys, data


def pad_ragged(layout: HeffLayout, name: str, keys, data, exts):
    """Zero-pad ragged blocks into the uniform reference layout (host arrays)."""
    dims = layout.dims[name]
    P = len(dims) - layout.n2[name]
    tail = dims[P:]
    blk = int(np.prod(tail))
    out = np.zeros(len(keys) * blk)
    off = 0
    for i, e in enumerate(exts):
        n = int(np.prod(e))
        b = np.zeros(tail)
        b[tuple(slice(0, x) for x in e)] = data[off: off + n].reshape(e, order="F")
        out[i * blk:(i + 1) * blk] = b.reshape(-1, order="F")
        off += n
    return out


def split_two_site(layout: HeffLayout, keys, data, exts, maxdim: int = 2 ** 62, cutoff: float = 0.0,
                   absorb: str = "right"):
    """Two-site tensor ψ[(ql, s1, s2, qr) | (ml, mr)] (ragged host triple) →
    A[(ql, s1, qc) | (ml, mc)] · B[(qc, s2, qr) | (mc, mr)], the U(1) split of a
    two-site DMRG step.

    Rows (ql, s1, ml) and columns (s2, qr, mr) are grouped by the charge c of
    the bond between the sites, Q(ql) + σ(s1) = Q(qr) − σ(s2); one SVD per
    charge; the singular values of all charges are truncated together: keep at
    most ``maxdim`` of them and drop the smallest as long as the dropped weight
    Σ s² / Σ s² stays ≤ ``cutoff`` (at least one is kept).  ``absorb="right"``
    gives a left-orthonormal A and B = S·V†; ``"left"`` gives A = U·S and a
    right-orthonormal B.  Returns (A, B, link, svals, truncerr) with A and B as
    (keys, data, exts) in the "A" layout of ``HeffLayout(left, link)`` and
    ``HeffLayout(link, right)`` (keys column-major sorted), ``link`` the new
    bond's sectors, ``svals`` the kept singular values (descending) and
    ``truncerr`` the dropped weight."""
    if absorb not in ("left", "right"):
        raise ValueError("absorb must be 'left' or 'right'")
    left, right = layout.left, layout.right
    blocks, off = {}, 0
    for k, e in zip(keys, exts):
        n = int(np.prod(e))
        blocks[tuple(k)] = np.asarray(data[off: off + n]).reshape(e, order="F")
        off += n
    rows, cols = {}, {}
    for (ql, s1, s2, qr) in blocks:
        c = left.charges[ql - 1] + PHYS[s1 - 1]
        rows.setdefault(c, set()).add((ql, s1))
        cols.setdefault(c, set()).add((s2, qr))
    svd = {}
    for c in sorted(rows):
        rseg = sorted(rows[c], key=lambda x: (x[1], x[0]))
        cseg = sorted(cols[c], key=lambda x: (x[1], x[0]))
        roff, coff, r0, c0 = {}, {}, 0, 0
        for ql, s1 in rseg:
            roff[(ql, s1)] = r0
            r0 += left.dims[ql - 1]
        for s2, qr in cseg:
            coff[(s2, qr)] = c0
            c0 += right.dims[qr - 1]
        M = np.zeros((r0, c0))
        for (ql, s1, s2, qr), b in blocks.items():
            if left.charges[ql - 1] + PHYS[s1 - 1] != c:
                continue
            r, cc = roff[(ql, s1)], coff[(s2, qr)]
            M[r: r + b.shape[0], cc: cc + b.shape[1]] = b
        U, S, Vt = np.linalg.svd(M, full_matrices=False)
        svd[c] = (U, S, Vt, rseg, roff, cseg, coff)
    allsv = sorted(((float(sv), c, i) for c, (U, S, Vt, *_r) in svd.items() for i, sv in enumerate(S)),
                   key=lambda t: (-t[0], t[1], t[2]))
    w = np.array([t[0] ** 2 for t in allsv])
    total = float(w.sum())
    m = len(allsv)
    if total > 0.0 and cutoff > 0.0:
        tail = np.cumsum(w[::-1])[::-1]  # tail[i] = weight of values i..end
        m = next((i for i in range(1, len(allsv) + 1) if i == len(allsv) or tail[i] <= cutoff * total), m)
    m = max(1, min(m, maxdim, len(allsv)))
    kept = {}
    for sv, c, i in allsv[:m]:
        kept[c] = kept.get(c, 0) + 1
    charges = sorted(kept)
    link = U1Link(charges, [kept[c] for c in charges])
    A_blocks, B_blocks = {}, {}
    for qc, c in enumerate(charges, start=1):
        U, S, Vt, rseg, roff, cseg, coff = svd[c]
        k = kept[c]
        Uk, Sk, Vk = U[:, :k], S[:k], Vt[:k, :]
        if absorb == "right":
            Vk = Sk[:, None] * Vk
        else:
            Uk = Uk * Sk[None, :]
        for ql, s1 in rseg:
            r = roff[(ql, s1)]
            A_blocks[(ql, s1, qc)] = Uk[r: r + left.dims[ql - 1], :]
        for s2, qr in cseg:
            cc = coff[(s2, qr)]
            B_blocks[(qc, s2, qr)] = Vk[:, cc: cc + right.dims[qr - 1]]

    def pack(bl):
        ks = sorted(bl, key=lambda k: k[::-1])
        return (ks, np.concatenate([bl[k].reshape(-1, order="F") for k in ks]) if ks else np.zeros(0),
                [bl[k].shape for k in ks])

    return pack(A_blocks), pack(B_blocks), link, np.array([t[0] for t in allsv[:m]]), float(w[m:].sum())


def _device_view(t):
    """The device payload of library tensor ``t`` as a torch float64 vector (no copy)."""
    import torch
    ptr, n = t.device_ptr()

    class _Payload:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                    "stream": None}

    return torch.as_tensor(_Payload(), device=f"cuda:{t.ctx.device}")


def split_two_site_device(layout: HeffLayout, psi, maxdim: int = 2 ** 62, cutoff: float = 0.0,
                          absorb: str = "right", method: str = "svd"):
    """``split_two_site`` on the device: the same grouping by centre charge,
    truncation rule and output layout, with the matrices assembled from the
    library tensor ``psi``'s device payload and factorised on the GPU in FP64
    (only the singular values travel to the host for the global truncation).
    Returns (A, B, link, svals, truncerr) with A and B library tensors in the
    "A" layout of ``HeffLayout(left, link)`` and ``HeffLayout(link, right)``.

    ``method``: "svd" (torch.linalg.svd of each centre-charge matrix M, as the
    reference's blocksparse_svd), or "gram": the density-matrix decomposition
    (ITensors' ``factorize(...; which_decomp="eigen")``): the eigenvectors of
    M M^T (absorb "right") or M^T M (absorb "left") by torch.linalg.eigh give
    the isometry, the singular values are the square roots of the eigenvalues,
    and the other factor is the projection U^T M (or M V), so A B is exactly
    the projection of psi on the kept states.  The eigenvalues carry an
    absolute error of order eps * sigma_max^2, well below a truncation cutoff
    on the discarded weight; singular values under about 1e-8 sigma_max are
    not resolved."""
    import torch
    import sparsebackends_b200 as sb
    if absorb not in ("left", "right"):
        raise ValueError("absorb must be 'left' or 'right'")
    if method not in ("svd", "gram"):
        raise ValueError("method must be 'svd' or 'gram'")
    ctx = psi.ctx
    left, right = layout.left, layout.right
    keys = [tuple(k) for k in psi.keys]
    exts = [tuple(int(x) for x in e) for e in psi.block_dims]
    offs = np.concatenate([[0], np.cumsum([e[0] * e[1] for e in exts])]).astype(np.int64)
    rows, cols = {}, {}
    for (ql, s1, s2, qr) in keys:
        c = left.charges[ql - 1] + PHYS[s1 - 1]
        rows.setdefault(c, set()).add((ql, s1))
        cols.setdefault(c, set()).add((s2, qr))
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{ctx.device}")
    svd = {}
    with torch.cuda.stream(stream):
        flat = _device_view(psi)
        for c in sorted(rows):
            rseg = sorted(rows[c], key=lambda x: (x[1], x[0]))
            cseg = sorted(cols[c], key=lambda x: (x[1], x[0]))
            roff, coff, r0, c0 = {}, {}, 0, 0
            for ql, s1 in rseg:
                roff[(ql, s1)] = r0
                r0 += left.dims[ql - 1]
            for s2, qr in cseg:
                coff[(s2, qr)] = c0
                c0 += right.dims[qr - 1]
            M = torch.zeros((r0, c0), dtype=torch.float64, device=flat.device)
            for i, (ql, s1, s2, qr) in enumerate(keys):
                if left.charges[ql - 1] + PHYS[s1 - 1] != c:
                    continue
                dl, dr = exts[i]
                r, cc = roff[(ql, s1)], coff[(s2, qr)]
                M[r: r + dl, cc: cc + dr] = flat[offs[i]: offs[i + 1]].view(dr, dl).t()
            if method == "svd":
                U, S, Vh = torch.linalg.svd(M, full_matrices=False)
            else:
                r = min(r0, c0)
                if absorb == "right":
                    lam, U = torch.linalg.eigh(M @ M.t())
                    U, Vh = U.flip(1)[:, :r], None
                else:
                    lam, V = torch.linalg.eigh(M.t() @ M)
                    U, Vh = None, V.flip(1)[:, :r].t()
                S = lam.flip(0)[:r].clamp_min(0.0).sqrt()
            svd[c] = (U, S, Vh, rseg, roff, cseg, coff, M)
        shost = {c: v[1].cpu().numpy() for c, v in svd.items()}
    allsv = sorted(((float(sv), c, i) for c, S in shost.items() for i, sv in enumerate(S)),
                   key=lambda t: (-t[0], t[1], t[2]))
    w = np.array([t[0] ** 2 for t in allsv])
    total = float(w.sum())
    m = len(allsv)
    if total > 0.0 and cutoff > 0.0:
        tail = np.cumsum(w[::-1])[::-1]
        m = next((i for i in range(1, len(allsv) + 1) if i == len(allsv) or tail[i] <= cutoff * total), m)
    m = max(1, min(m, maxdim, len(allsv)))
    kept = {}
    for sv, c, i in allsv[:m]:
        kept[c] = kept.get(c, 0) + 1
    charges = sorted(kept)
    link = U1Link(charges, [kept[c] for c in charges])
    A_blocks, B_blocks = {}, {}
    with torch.cuda.stream(stream):
        for qc, c in enumerate(charges, start=1):
            U, S, Vh, rseg, roff, cseg, coff, M = svd[c]
            k = kept[c]
            if method == "gram":
                if absorb == "right":
                    Uk = U[:, :k]
                    Vk = Uk.t() @ M
                else:
                    Vk = Vh[:k, :]
                    Uk = M @ Vk.t()
            else:
                Uk, Sk, Vk = U[:, :k], S[:k], Vh[:k, :]
                if absorb == "right":
                    Vk = Sk[:, None] * Vk
                else:
                    Uk = Uk * Sk[None, :]
            for ql, s1 in rseg:
                r = roff[(ql, s1)]
                A_blocks[(ql, s1, qc)] = Uk[r: r + left.dims[ql - 1], :]
            for s2, qr in cseg:
                cc = coff[(s2, qr)]
                B_blocks[(qc, s2, qr)] = Vk[:, cc: cc + right.dims[qr - 1]]

    def make(bl, lo: U1Link, hi: U1Link):
        ks = sorted(bl, key=lambda k: k[::-1])
        ex = [tuple(bl[k].shape) for k in ks]
        n = int(sum(a * b for a, b in ex))
        t = sb.NewBlockSparseSorted((lo.S, 2, hi.S, lo.D, hi.D), 2, ks, None, np.zeros(max(n, 1))[:n], ctx=ctx,
                                    block_dims=ex)
        if n:
            with torch.cuda.stream(stream):
                view = _device_view(t)
                o = 0
                for k, e in zip(ks, ex):
                    view[o: o + e[0] * e[1]] = bl[k].t().reshape(-1)  # column-major block
                    o += e[0] * e[1]
        return t

    A = make(A_blocks, left, link)
    B = make(B_blocks, link, right)
    stream.synchronize()
    return A, B, link, np.array([t[0] for t in allsv[:m]]), float(w[m:].sum())


def _channel_conj(layout: HeffLayout, qw: int) -> int:
    """1-based sector index of the conjugate MPO channel sector (charge -c)."""
    w = layout.mpo
    return w.index(-w.charges[qw - 1]) + 1


def hermitian_operators(layout: HeffLayout, rng: np.random.Generator, scales=None):
    """Seeded L, W1, W2, R (ragged host triples (keys, data, block_dims)) for
    which the two-site H_eff is a real symmetric operator.

    With the channel involution w -> w' (charge c -> -c, same index inside the
    sector) it suffices that L[a', w, a] = L[a, w', a'], R likewise and
    W[wl, s', s, wr] = W[wl', s, s', wr']: substituting w -> w' in the sum over
    channels then swaps bra and ket.  Each operator is the average of a random
    one and its transpose under that map; the charge rules map allowed keys to
    allowed keys.  Requires a charge-symmetric MPO link."""
    w = layout.mpo
    for q, dq in zip(w.charges, w.dims):
        if -q not in w.charges or w.dims[w.index(-q)] != dq:
            raise ValueError("hermitian_operators needs an MPO link symmetric under c -> -c")
    scales = scales or {"L": 0.05, "W1": 0.3, "W2": 0.3, "R": 0.05}
    out = {}
    for name in ("L", "W1", "W2", "R"):
        keys, data, exts = random_block_tensor(layout, name, rng, scales[name], ragged=True)
        blocks, off = {}, 0
        for k, e in zip(keys, exts):
            n = int(np.prod(e))
            blocks[k] = data[off: off + n].reshape(e, order="F")
            off += n
        sym = []
        for k, e in zip(keys, exts):
            if name in ("L", "R"):
                kt = (k[2], _channel_conj(layout, k[1]), k[0])
                bt = np.transpose(blocks[kt], (2, 1, 0))
            else:
                kt = (_channel_conj(layout, k[0]), k[2], k[1], _channel_conj(layout, k[3]))
                bt = blocks[kt]
            sym.append((0.5 * (blocks[k] + bt)).reshape(-1, order="F"))
        out[name] = (keys, np.concatenate(sym) if sym else np.zeros(0), exts)
    return out


class HeffOperator:
    """x -> H_eff x as a new device tensor (the operator KrylovKit's eigsolve
    applies: ITensorMPS ``product(::ProjMPO, v)``).  Operands stay resident;
    each call runs the contraction chain and copies the result out of the
    chain's reused output buffer."""

    def __init__(self, layout: HeffLayout, L, W1, W2, R, ctx=None, graph_like=None, w12: bool = False,
                 precision: str = "f64", f32_intermediates: bool = None):
        """With ``graph_like`` (a vector with the layout of the inputs to come)
        the chain is captured once as a CUDA graph on a private input buffer;
        each call copies its input there and replays the graph.  ``w12`` picks
        the chain ψ·L·(W1·W2)·R (``HeffChain``).  ``precision``: the context
        precision the chain's block GEMMs run in (``Context.set_precision``;
        set for each apply and restored after it); in a tensor-core precision
        the intermediates are FP32 unless ``f32_intermediates`` is False."""
        import sparsebackends_b200 as sb
        self.sb = sb
        self.ctx = ctx or L.ctx
        self.precision = precision
        # relative accuracy of one apply (krylov.eigsolve's optol): measured
        # per-block errors of the tensor-core GEMMs are a few 1e-7 to 1e-6
        # (3xTF32) and 3e-4 (TF32); the bound leaves a margin
        self.accuracy = {"f64": 0.0, "tf32x3": 1e-5, "tf32": 3e-2}[precision]
        if f32_intermediates is None:
            f32_intermediates = precision != "f64"
        self.chain = HeffChain(layout, self.ctx, w12=w12, f32_intermediates=f32_intermediates)
        self.ops = (L, W1, W2, R)
        self.calls = 0
        self.graph = None
        if graph_like is not None:
            self.x = sb.copy(graph_like)
            prev = self._enter()
            try:
                self.graph = self.chain.capture(self.x, *self.ops)
            finally:
                self._leave(prev)

    def _enter(self) -> str:
        prev = self.ctx.precision
        if prev != self.precision:
            self.ctx.set_precision(self.precision)
        return prev

    def _leave(self, prev: str) -> None:
        if prev != self.precision:
            self.ctx.set_precision(prev)

    def __call__(self, psi):
        self.calls += 1
        prev = self._enter()
        try:
            if self.graph is not None:
                self.sb.map_(self.x, psi, self.sb.MAP_COPY)
                self.graph.launch()
                return self.sb.copy(self.chain.out["T4"])
            return self.sb.copy(self.chain.apply(psi, *self.ops))
        finally:
            self._leave(prev)


def contract_new(labelsC, n2C, A, labelsA, B, labelsB):
    """``contract!`` into a freshly allocated block-sparse C whose dims follow
    from the operands' dims by label (the caller's allocation in
    tensor_wrappers.jl:654)."""
    import sparsebackends_b200 as sb
    ext = dict(zip(labelsA, A.dims))
    ext.update(zip(labelsB, B.dims))
    C = sb.NewBlockSparseSorted.empty(tuple(ext[x] for x in labelsC), n2C, ctx=A.ctx)
    return sb.contract_(C, labelsC, A, labelsA, B, labelsB)


# The three contract! calls of each environment update: (labels of the result,
# its tail count, labels of the left operand, labels of the right operand).
# make_L: E1 = L*A, E2 = E1*W, L' = E2*A;  make_R: F1 = R*B, F2 = F1*W, R' = F2*B.
MAKE_L_STEPS = (
    (["qlp", "qwl", "s1", "qr", "mr", "mlp", "mwl"], 3,
     ["qlp", "qwl", "ql", "mlp", "mwl", "ml"], ["ql", "s1", "qr", "ml", "mr"]),
    (["qlp", "qr", "s1p", "qwm", "mr", "mlp", "mwm"], 3,
     ["qlp", "qwl", "s1", "qr", "mr", "mlp", "mwl"], ["qwl", "s1p", "s1", "qwm", "mwl", "mwm"]),
    (["qrp", "qwm", "qr", "mrp", "mwm", "mr"], 3,
     ["qlp", "qr", "s1p", "qwm", "mr", "mlp", "mwm"], ["qlp", "s1p", "qrp", "mlp", "mrp"]),
)
MAKE_R_STEPS = (
    (["qrp", "qwm", "ql", "s1", "ml", "mrp", "mwm"], 3,
     ["qrp", "qwm", "qr", "mrp", "mwm", "mr"], ["ql", "s1", "qr", "ml", "mr"]),
    (["qrp", "ql", "s1p", "qwl", "ml", "mrp", "mwl"], 3,
     ["qrp", "qwm", "ql", "s1", "ml", "mrp", "mwm"], ["qwl", "s1p", "s1", "qwm", "mwl", "mwm"]),
    (["qlp", "qwl", "ql", "mlp", "mwl", "ml"], 3,
     ["qrp", "ql", "s1p", "qwl", "ml", "mrp", "mwl"], ["qlp", "s1p", "qrp", "mlp", "mrp"]),
)


def _env_update(steps, E, A, W):
    (c1, n1, la1, lb1), (c2, n2, la2, lb2), (c3, n3, la3, lb3) = steps
    E1 = contract_new(c1, n1, E, la1, A, lb1)
    E2 = contract_new(c2, n2, E1, la2, W, lb2)
    return contract_new(c3, n3, E2, la3, A, lb3)


def make_L(L, A, W):
    """Left environment update, ITensorMPS ``makeL!``: L' = L · A · W · Ā.

    L'[(qr', mr'), (qw', mw'), (qr, mr)] = sum L[(ql', ml'), (qw, mw), (ql, ml)]
    A[(ql, ml), s, (qr, mr)] W[(qw, mw), s', s, (qw', mw')] A[(ql', ml'), s', (qr', mr')]
    as three ``contract!`` calls on the device (real tensors: Ā = A).  The
    result has the layout of the environments (labels q', qw, q | m', mw, m)."""
    return _env_update(MAKE_L_STEPS, L, A, W)


def make_R(R, B, W):
    """Right environment update, ITensorMPS ``makeR!``: R' = R · B · W · B̄.

    R'[(ql', ml'), (qw, mw), (ql, ml)] = sum R[(qr', mr'), (qw', mw'), (qr, mr)]
    B[(ql, ml), s, (qr, mr)] W[(qw, mw), s', s, (qw', mw')] B[(ql', ml'), s', (qr', mr')]."""
    return _env_update(MAKE_R_STEPS, R, B, W)


class HeffChain:
    """Two-site H_eff · ψ through ``contract!`` calls on the device.

    The default order is ITensorMPS ``product(::ProjMPO, v)``'s: ψ·L, ·W1, ·W2,
    ·R (four contractions).  With ``w12=True`` the two MPO tensors are
    contracted with each other first, W12 = W1·W2 (a contraction of MPO blocks
    only, recomputed by every apply), and ψ·L·W12·R takes three: the same
    FLOPs in the MPO steps, with the T2 intermediate never written or read.

    The intermediate and output tensors are allocated once and overwritten by
    every apply (``contract!`` semantics)."""

    STEPS = (("T1", "L", "psi"), ("T2", "T1", "W1"), ("T3", "T2", "W2"), ("T4", "R", "T3"))
    STEPS_W12 = (("W12", "W1", "W2"), ("T1", "L", "psi"), ("T3", "T1", "W12"), ("T4", "R", "T3"))

    def __init__(self, layout: HeffLayout, ctx=None, w12: bool = False, f32_intermediates: bool = False):
        """``f32_intermediates``: T1, T2, T3 (and W12) are stored in FP32
        (sb_tensor_create_bs_f32), for a context in a tensor-core precision:
        the MPO steps then move half the bytes; T4 stays FP64."""
        import sparsebackends_b200 as sb
        self.sb = sb
        self.layout = layout
        self.steps = self.STEPS_W12 if w12 else self.STEPS
        self.out = {n: sb.NewBlockSparseSorted.empty(layout.dims[n], layout.n2[n], ctx=ctx,
                                                     f32=f32_intermediates and n not in ("T4", "W12"))
                    for n in {c for c, _, _ in self.steps}}

    def apply(self, psi, L, W1, W2, R):
        t = {"psi": psi, "L": L, "W1": W1, "W2": W2, "R": R, **self.out}
        lab = self.layout.labels
        for c, a, b in self.steps:
            self.sb.contract_(t[c], lab[c], t[a], lab[a], t[b], lab[b])
        return self.out["T4"]

    def capture(self, psi, L, W1, W2, R):
        """Run the chain once, then capture it as one CUDA graph bound to these
        tensors.  ``graph.launch()`` recomputes ``self.out["T4"]`` from the
        current values of ``psi`` (and of the operators): the per-call host
        planning and plan uploads are paid once, at capture."""
        self.apply(psi, L, W1, W2, R)
        return psi.ctx.capture(lambda: self.apply(psi, L, W1, W2, R),
                               keep=[psi, L, W1, W2, R, *self.out.values()])


GRADE = {"ml": "ql", "mlp": "qlp", "mr": "qr", "mrp": "qrp", "mwl": "qwl", "mwm": "qwm", "mwr": "qwr"}


def _link_of(layout: HeffLayout, qlabel: str) -> U1Link:
    if qlabel in ("ql", "qlp"):
        return layout.left
    if qlabel in ("qr", "qrp"):
        return layout.right
    return layout.mpo


def chain_structure(layout: HeffLayout, steps=HeffChain.STEPS):
    """Key-level simulation of the chain's steps: per step the matched block
    pairs (as label->value dicts) and the output key set.  Pure integer work on
    the host; used for FLOP accounting only."""
    lab = layout.labels
    keys = {n: [dict(zip(lab[n][: len(lab[n]) - layout.n2[n]], k)) for k in layout.keys[n]]
            for n in ("psi", "L", "W1", "W2", "R")}
    out = []
    for c, a, b in steps:
        la, lb, lc = lab[a], lab[b], lab[c]
        Pa, Pb, Pc = (len(x) - layout.n2[n] for x, n in ((la, a), (lb, b), (lc, c)))
        shared_pref = [x for x in la[:Pa] if x in lb[:Pb]]
        groups = {}
        for kb in keys[b]:
            groups.setdefault(tuple(kb[x] for x in shared_pref), []).append(kb)
        pairs, ckeys = [], {}
        for ka in keys[a]:
            for kb in groups.get(tuple(ka[x] for x in shared_pref), []):
                kv = {**ka, **kb}
                pairs.append(kv)
                ckeys[tuple(kv[x] for x in lc[:Pc])] = {x: kv[x] for x in lc[:Pc]}
        keys[c] = list(ckeys.values())
        red = [x for x in la[Pa:] if x in lb[Pb:]]
        keepA = [x for x in la[Pa:] if x not in red]
        keepB = [x for x in lb[Pb:] if x not in red]
        out.append(dict(C=c, A=a, B=b, pairs=pairs, nC=len(keys[c]), red=red, keepA=keepA, keepB=keepB))
    return out


def chain_flops(layout: HeffLayout, padded: bool = True, steps=HeffChain.STEPS) -> float:
    """FLOPs of one H_eff apply: the sum over matched block pairs of 2·m·n·k.

    ``padded=True`` counts the executed (zero-padded) GEMM shapes;
    ``padded=False`` counts the unpadded sector extents, the algorithmic work."""
    total = 0.0
    for st in chain_structure(layout, steps):
        for kv in st["pairs"]:
            def ext(x):
                if padded:
                    return layout.ext[x]
                q = GRADE[x]
                return _link_of(layout, q).dims[kv[q] - 1]
            m = np.prod([ext(x) for x in st["keepA"]]) if st["keepA"] else 1
            n = np.prod([ext(x) for x in st["keepB"]]) if st["keepB"] else 1
            k = np.prod([ext(x) for x in st["red"]]) if st["red"] else 1
            total += 2.0 * m * n * k
    return total
