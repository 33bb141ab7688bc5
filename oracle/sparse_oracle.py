"""CPU restatement of SparseBackends' block-sparse contraction path (numpy).

THIS MODULE IS TEST INFRASTRUCTURE.  It is the parity oracle for the CUDA
library in ``sparsebackends_b200``: only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may import it.  The product path never
calls it.

It restates, function by function, the Julia reference (paths relative to the
``SparseBackends`` package):

* storage      ``src/blocksparse/storage.jl``, ``src/coo/storage.jl``,
               ``src/aliased/storage.jl`` and their ``conversions.jl``
* dispatch     ``src/tensoralgebra/contract.jl:37-104``
* kernels      ``src/tensoralgebra/contract_{coo,coo_dense,coo_bs,bs_bs,bs_dense}.jl``,
               ``contract_aliased_coo_dense.jl``, ``contract_aliased.jl``,
               ``contract_aliased_shared.jl``

Conventions kept from the reference:
* keys are 1-based integer tuples; block-sparse and aliased keys are sorted by
  the column-major linear index of the prefix (``_prefix_lin``);
* payloads are flat column-major (Fortran) vectors;
* C is overwritten by every kernel; block existence rules (structural or
  value dependent) are reproduced exactly;
* elementwise update order and rounding (``c += a*b`` without fusion, Kahan
  compensation) follow the reference, so hand-loop kernels are bit-exact;
  BLAS calls (``mul!``, ``ger!``) are numpy ``@`` / ``outer``.

Dense operands are numpy arrays indexed like the Julia arrays (0-based);
reshapes that the reference does on column-major memory use ``order='F'``.

Parity pinning: the reference cannot run here (no Julia); this restatement is
pinned by the reference's own known-answer tests (``SparseBackends/test/**``),
restated in ``tests/test_oracle_kat.py``.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field
from typing import Any, Dict, List, Sequence, Tuple

import numpy as np

Key = Tuple[int, ...]


class OracleError(Exception):
    """Mirrors Julia's ErrorException/AssertionError raised by the reference."""


def _assert(cond: bool, msg: str = "assertion failed") -> None:
    if not cond:
        raise OracleError(msg)


def _prod(xs) -> int:
    p = 1
    for x in xs:
        p *= int(x)
    return p


def prefix_lin(k: Sequence[int], pdims: Sequence[int]) -> int:
    """``_prefix_lin`` (src/blocksparse/storage.jl:16-18): 1-based column-major."""
    idx, stride = 1, 1
    for d in range(len(pdims)):
        idx += (int(k[d]) - 1) * stride
        stride *= int(pdims[d])
    return idx


def _sortperm(keys: Sequence[Any], by) -> List[int]:
    # Julia's default sortperm is stable; Python's sort is stable too.
    return sorted(range(len(keys)), key=lambda i: by(keys[i]))


# ───────────────────────────── storage types ──────────────────────────────


class BS:
    """``NewBlockSparseSorted`` (src/blocksparse/storage.jl:3-9).

    Payload slots are kept as a list of per-id arrays so that appending a
    block is O(blksize), like Julia's amortised ``append!`` (storage.jl:67-71);
    ``data`` concatenates them on demand."""

    def __init__(self, dims, n2, keys=None, ids=None, data=None):
        self.dims = tuple(int(d) for d in dims)
        self.n2 = int(n2)
        self.keys: List[Key] = list(keys or [])
        self.ids: List[int] = list(ids or [])
        self.data = np.zeros(0) if data is None else data

    @property
    def data(self) -> np.ndarray:
        if not self._slots:
            return np.zeros(0)
        return np.concatenate(self._slots)

    @data.setter
    def data(self, value) -> None:
        v = np.asarray(value, dtype=np.float64).reshape(-1)
        b = self.blksize
        self._slots = [v[i * b:(i + 1) * b].copy() for i in range(len(v) // b)] if b else []

    @property
    def N(self) -> int:
        return len(self.dims)

    @property
    def P(self) -> int:
        return len(self.dims) - self.n2

    @property
    def blksize(self) -> int:
        return _prod(self.dims[self.P:])

    @staticmethod
    def empty(dims, n2) -> "BS":
        dims = tuple(int(d) for d in dims)
        _assert((len(dims) == 0 and n2 == 0) or (0 < n2 <= len(dims)))
        _assert(all(d >= 1 for d in dims))
        return BS(dims, n2)

    def block(self, id_: int) -> np.ndarray:
        """``_block_view`` (storage.jl:138-141); id is 1-based; writes go through."""
        return self._slots[id_ - 1]

    def find_key(self, k: Key) -> Tuple[int, bool]:
        """``_find_key`` (storage.jl:49-65) → (0-based insert position, found)."""
        pd = self.dims[: self.P]
        target = prefix_lin(k, pd)
        lo, hi = 0, len(self.keys)
        while lo < hi:
            mid = (lo + hi) >> 1
            if prefix_lin(self.keys[mid], pd) < target:
                lo = mid + 1
            else:
                hi = mid
        found = lo < len(self.keys) and self.keys[lo] == k
        return lo, found

    def ensure_block(self, k: Key) -> int:
        """``_ensure_block!`` (storage.jl:73-83): sorted insert + zero append."""
        i, found = self.find_key(k)
        if found:
            return self.ids[i]
        self._slots.append(np.zeros(self.blksize))
        id_ = len(self._slots)
        self.keys.insert(i, k)
        self.ids.insert(i, id_)
        return id_

    def clear(self) -> None:
        self.keys, self.ids, self._slots = [], [], []

    def blocks_by_key(self) -> Dict[Key, np.ndarray]:
        return {k: self.block(i).copy() for k, i in zip(self.keys, self.ids)}

    def getindex(self, *I) -> float:
        P = self.P
        k = tuple(I[:P])
        i, found = self.find_key(k)
        if not found:
            return 0.0
        lin = 0
        stride = 1
        for j in range(self.n2):
            lin += (I[P + j] - 1) * stride
            stride *= self.dims[P + j]
        return float(self.block(self.ids[i])[lin])

    def setindex(self, v, *I) -> None:
        P = self.P
        id_ = self.ensure_block(tuple(I[:P]))
        lin = 0
        stride = 1
        for j in range(self.n2):
            lin += (I[P + j] - 1) * stride
            stride *= self.dims[P + j]
        self.block(id_)[lin] = v


@dataclass
class COO:
    """``COOTensor`` (src/coo/storage.jl:1-6)."""

    dims: Tuple[int, ...]
    keys: List[Key] = field(default_factory=list)
    vals: List[float] = field(default_factory=list)
    dirty: bool = False

    @property
    def N(self) -> int:
        return len(self.dims)


@dataclass
class Aliased:
    """``AliasedBlockSparse`` (src/aliased/storage.jl:46-54)."""

    dims: Tuple[int, ...]
    n2: int
    templates: np.ndarray = field(default_factory=lambda: np.zeros(0))
    n_templates: int = 0
    keys: List[Key] = field(default_factory=list)
    alias_ids: List[int] = field(default_factory=list)
    scalars: List[float] = field(default_factory=list)

    @property
    def N(self) -> int:
        return len(self.dims)

    @property
    def P(self) -> int:
        return len(self.dims) - self.n2

    @property
    def blksize(self) -> int:
        return _prod(self.dims[self.P:])

    @staticmethod
    def empty(dims, n2) -> "Aliased":
        dims = tuple(int(d) for d in dims)
        _assert(0 < n2 <= len(dims))
        return Aliased(dims, n2)

    def template(self, t: int) -> np.ndarray:
        b = self.blksize
        return self.templates[(t - 1) * b: t * b]

    def clear(self) -> None:
        self.templates = np.zeros(0)
        self.n_templates = 0
        self.keys, self.alias_ids, self.scalars = [], [], []

    def logical_blocks(self) -> Dict[Key, np.ndarray]:
        """Per-key logical block ``scalar * template`` (the comparison unit)."""
        return {k: s * self.template(t) for k, t, s in zip(self.keys, self.alias_ids, self.scalars)}


def is_dense_array(x) -> bool:
    return isinstance(x, np.ndarray)


def dims_of(x) -> Tuple[int, ...]:
    return tuple(x.shape) if is_dense_array(x) else tuple(x.dims)


# ───────────────────────────── conversions ────────────────────────────────


def blocksparse_from_dense(A: np.ndarray, n2: int, atol=0.0, rtol=0.0, dropzeros=True) -> BS:
    """``blocksparse_from_dense`` (src/blocksparse/conversions.jl:21-75)."""
    A = np.asarray(A, dtype=np.float64)
    N = A.ndim
    _assert(0 <= n2 <= N)
    P = N - n2
    dims = tuple(A.shape)
    gmax = 0.0 if rtol == 0 else (float(np.max(np.abs(A))) if A.size else 0.0)
    tol = max(atol, rtol * gmax)
    out = BS(dims, n2, [], [], np.zeros(0))
    blocks = []
    # CartesianIndices(prefix_dims) iterates column-major (first index fastest)
    pdims = dims[:P]
    for lin in range(_prod(pdims)):
        pref = np.unravel_index(lin, pdims, order="F") if P else ()
        sub = A[tuple(int(p) for p in pref)]
        buf = np.asarray(sub).reshape(-1, order="F")
        bmax = float(np.max(np.abs(buf))) if buf.size else 0.0
        if (not dropzeros) or bmax > tol:
            out.keys.append(tuple(int(p) + 1 for p in pref))
            out.ids.append(len(out.keys))
            blocks.append(buf.copy())
    out.data = np.concatenate(blocks) if blocks else np.zeros(0)
    return out


def bs_is_dense(A: BS) -> bool:
    """``is_dense`` (src/blocksparse/storage.jl:413-425)."""
    if A.P == 0:
        _assert(len(A.keys) <= 1, "P=0 means no prefix, so at most one block (the whole tensor) is allowed")
        return True
    return len(A.keys) == _prod(A.dims[: A.P])


def bs_to_dense(B: BS) -> np.ndarray:
    """``to_dense(::NewBlockSparseSorted)`` (conversions.jl:83-187), no merge."""
    out = np.zeros(B.dims)
    P = B.P
    tdims = B.dims[P:]
    for k, i in zip(B.keys, B.ids):
        out[tuple(x - 1 for x in k)] = B.block(i).reshape(tdims, order="F")
    return out


def coo_from_dense(A: np.ndarray, atol=1e-12, rtol=0.0) -> COO:
    """``coo_from_dense`` (src/coo/conversions.jl:13-26): col-major scan."""
    A = np.asarray(A, dtype=np.float64)
    keys, vals = [], []
    flat = A.reshape(-1, order="F")
    for lin, v in enumerate(flat):
        if abs(v) > atol + rtol * abs(v):
            keys.append(tuple(int(x) + 1 for x in np.unravel_index(lin, A.shape, order="F")))
            vals.append(float(v))
    return COO(tuple(A.shape), keys, vals, False)


def coo_to_dense(A: COO) -> np.ndarray:
    out = np.zeros(A.dims)
    for k, v in zip(A.keys, A.vals):
        out[tuple(x - 1 for x in k)] = v
    return out


def aliased_to_blocksparse(A: Aliased) -> BS:
    """``to_blocksparse`` (src/aliased/conversions.jl:18-32)."""
    out = BS(A.dims, A.n2, list(A.keys), list(range(1, len(A.keys) + 1)), np.zeros(0))
    parts = [s * A.template(t) for t, s in zip(A.alias_ids, A.scalars)]
    out.data = np.concatenate(parts) if parts else np.zeros(0)
    return out


def aliased_to_dense(A: Aliased) -> np.ndarray:
    return bs_to_dense(aliased_to_blocksparse(A))


def aliased_from_blocksparse_unique(B: BS) -> Aliased:
    """Build an aliased tensor whose blocks each own one template (scalar 1).

    Used by tests to feed the aliased kernels; identical payloads are shared
    so that the template bookkeeping is exercised.
    """
    out = Aliased.empty(B.dims, B.n2)
    seen: Dict[bytes, int] = {}
    tmpl = []
    for k, i in zip(B.keys, B.ids):
        blk = B.block(i)
        h = blk.tobytes()
        if h not in seen:
            tmpl.append(blk.copy())
            seen[h] = len(tmpl)
        out.keys.append(k)
        out.alias_ids.append(seen[h])
        out.scalars.append(1.0)
    out.templates = np.concatenate(tmpl) if tmpl else np.zeros(0)
    out.n_templates = len(tmpl)
    return out


# ───────────────────────────── permutes ───────────────────────────────────


def _check_no_cross_perm(perm: Sequence[int], N: int, P: int) -> None:
    """``_check_no_cross_perm`` (storage.jl:126-132); perm is 1-based."""
    _assert(len(perm) == N)
    _assert(sorted(perm) == list(range(1, N + 1)), "perm must be a permutation of 1:N")
    _assert(all(p <= P for p in perm[:P]), "No-cross reorder violated: output prefix axis uses old block axis")
    _assert(all(p > P for p in perm[P:]), "No-cross reorder violated: output block axis uses old prefix axis")


def _tail_permute(vec: np.ndarray, tdims_old: Sequence[int], perm_block: Sequence[int]) -> np.ndarray:
    """Gather a column-major block through ``map_old`` (storage.jl:220-261)."""
    if len(tdims_old) == 0:
        return vec.copy()
    arr = vec.reshape(tuple(tdims_old), order="F")
    return np.transpose(arr, [p - 1 for p in perm_block]).reshape(-1, order="F")


def bs_permutedims(A: BS, perm: Sequence[int]) -> BS:
    """``Base.permutedims(::NewBlockSparseSorted, perm)`` (storage.jl:188-264)."""
    perm = [int(p) for p in perm]
    N, P = A.N, A.P
    _check_no_cross_perm(perm, N, P)
    dimsB = tuple(A.dims[p - 1] for p in perm)
    perm_prefix = perm[:P]
    perm_block = [p - P for p in perm[P:]]
    newkeys = [tuple(k[j - 1] for j in perm_prefix) for k in A.keys]
    pd = dimsB[:P]
    p = _sortperm(newkeys, lambda k: prefix_lin(k, pd))
    out = BS(dimsB, A.n2, [newkeys[i] for i in p], list(range(1, len(p) + 1)), np.zeros(0))
    tdims_old = A.dims[P:]
    parts = [_tail_permute(A.block(A.ids[i]), tdims_old, perm_block) for i in p]
    out.data = np.concatenate(parts) if parts else np.zeros(0)
    return out


def coo_permutedims(A: COO, perm: Sequence[int]) -> COO:
    """``Base.permutedims(::COOTensor, perm)`` (coo/storage.jl:153-162): dirty."""
    perm = [int(p) for p in perm]
    _assert(sorted(perm) == list(range(1, A.N + 1)))
    dimsB = tuple(A.dims[p - 1] for p in perm)
    keys = [tuple(k[p - 1] for p in perm) for k in A.keys]
    return COO(dimsB, keys, list(A.vals), True)


def coo_sort(A: COO) -> COO:
    """``sort_coo!`` (coo/storage.jl:182-189): ``sortperm(keys; by=reverse)``."""
    if not A.dirty:
        return A
    p = _sortperm(A.keys, lambda k: tuple(reversed(k)))
    A.keys = [A.keys[i] for i in p]
    A.vals = [A.vals[i] for i in p]
    A.dirty = False
    return A


def aliased_permutedims(A: Aliased, perm: Sequence[int]) -> Aliased:
    """``Base.permutedims(::AliasedBlockSparse, perm)`` (aliased/storage.jl:172-236)."""
    perm = [int(p) for p in perm]
    N, P = A.N, A.P
    _check_no_cross_perm(perm, N, P)
    dimsB = tuple(A.dims[p - 1] for p in perm)
    perm_block = [p - P for p in perm[P:]]
    tdims_old = A.dims[P:]
    parts = [_tail_permute(A.template(t), tdims_old, perm_block) for t in range(1, A.n_templates + 1)]
    newkeys = [tuple(k[j - 1] for j in perm[:P]) for k in A.keys]
    pd = dimsB[:P]
    p = _sortperm(newkeys, lambda k: prefix_lin(k, pd))
    out = Aliased(dimsB, A.n2)
    out.templates = np.concatenate(parts) if parts else np.zeros(0)
    out.n_templates = A.n_templates
    out.keys = [newkeys[i] for i in p]
    out.alias_ids = [A.alias_ids[i] for i in p]
    out.scalars = [A.scalars[i] for i in p]
    return out


def dense_permutedims(B: np.ndarray, perm: Sequence[int]) -> np.ndarray:
    return np.ascontiguousarray(np.transpose(B, [int(p) - 1 for p in perm]))


# ───────────────────────────── helpers (contract_bs_bs.jl) ────────────────


def _outer_add(C: np.ndarray, a: np.ndarray, b: np.ndarray) -> None:
    """``_outer_add!`` (contract_bs_bs.jl:7-18): C[i + j*m] += a[i]*b[j]."""
    m, n = len(a), len(b)
    Cm = C.reshape((m, n), order="F")
    Cm += np.multiply.outer(a, b)


def _rank1_add(Cmat: np.ndarray, x: np.ndarray, y: np.ndarray) -> None:
    """``_rank1_add_blas!`` (contract_bs_bs.jl:118-124): BLAS ger, C += x yᵀ."""
    Cmat += np.multiply.outer(x, y)


def _cmat(vec: np.ndarray, m: int, n: int) -> np.ndarray:
    """Column-major (m, n) view of a flat block (writes go through)."""
    return vec.reshape((n, m)).T if vec.size else vec.reshape((m, n))


def _find_permutation_for_tensor(P: int, N: int, axisr: int) -> List[int]:
    """``_find_permutation_for_tensor`` (contract_bs_bs.jl:33-45); 1-based."""
    if axisr <= P:
        pref = [a for a in range(1, P + 1) if a != axisr] + [axisr]
        return pref + list(range(P + 1, N + 1))
    dense = [d for d in range(1, N - P + 1) if d != axisr - P] + [axisr - P]
    return list(range(1, P + 1)) + [P + d for d in dense]


def _permute_r_to_last_prefix(T: BS, labels: List[Any], rlab):
    """``_permute_r_to_last_prefix`` (contract_bs_bs.jl:77-95)."""
    axisr = labels.index(rlab) + 1
    _assert(axisr <= T.P, "rlab must be in prefix to use prefix kernel")
    if axisr == T.P:
        return T, labels
    perm = _find_permutation_for_tensor(T.P, T.N, axisr)
    return bs_permutedims(T, perm), [labels[p - 1] for p in perm]


def _cdense_grouping_and_orders(Cdense, keepA, keepB):
    """``_cdense_grouping_and_orders`` (contract_bs_bs.jl:470-505)."""
    sA, sB = set(keepA), set(keepB)
    origin = []
    for lab in Cdense:
        if lab in sA:
            origin.append(True)
        elif lab in sB:
            origin.append(False)
        else:
            raise OracleError(f"Cdense label {lab} not found in keepA/keepB")
    firstB = next((i for i, o in enumerate(origin) if not o), None)
    firstA = next((i for i, o in enumerate(origin) if o), None)
    lastA = max((i for i, o in enumerate(origin) if o), default=None)
    lastB = max((i for i, o in enumerate(origin) if not o), default=None)
    if firstB is None or firstA is None:
        mode = "AthenB"
    elif lastA < firstB:
        mode = "AthenB"
    elif lastB < firstA:
        mode = "BthenA"
    else:
        mode = "interleaved"
    return mode, [l for l in Cdense if l in sA], [l for l in Cdense if l in sB]


def _find_perm_A_join_dense(labelsA, PA, shared_prefix, desired_keepA, red_dense):
    """``_find_perm_for_A_join_and_dense_order`` (contract_bs_bs.jl:513-536)."""
    pos = {l: i + 1 for i, l in enumerate(labelsA)}
    sp = [pos[l] for l in shared_prefix]
    keep_pref = [a for a in range(1, PA + 1) if a not in set(sp)]
    keep_axes = [pos[l] - PA for l in desired_keepA]
    red_axes = [pos[l] - PA for l in red_dense]
    _assert(len(keep_axes) + len(red_axes) == len(labelsA) - PA)
    return keep_pref + sp + [PA + d for d in keep_axes + red_axes]


def _find_perm_B_join_dense_redfirst(labelsB, PB, shared_prefix, red_dense, desired_keepB):
    """``_find_perm_for_B_join_and_dense_redfirst_order`` (contract_bs_bs.jl:544-567)."""
    pos = {l: i + 1 for i, l in enumerate(labelsB)}
    sp = [pos[l] for l in shared_prefix]
    keep_pref = [a for a in range(1, PB + 1) if a not in set(sp)]
    red_axes = [pos[l] - PB for l in red_dense]
    keep_axes = [pos[l] - PB for l in desired_keepB]
    _assert(len(red_axes) + len(keep_axes) == len(labelsB) - PB)
    return keep_pref + sp + [PB + d for d in red_axes + keep_axes]


def _advance_run(keys: List[Key], i0: int, n: int, pos: List[int]) -> int:
    """``_advance_run`` (contract_bs_bs.jl:455-464), 0-based, exclusive end."""
    if not pos:
        return n
    k0 = keys[i0]
    i = i0 + 1
    while i < n and all(k0[p - 1] == keys[i][p - 1] for p in pos):
        i += 1
    return i


# Order in which the merge-join compares the join tuples of two keys.
# "sorted" (default): from the last join axis down, the order the keys are
# sorted in.  "reference": from the first join axis up, exactly as
# ``_cmp_join_tuple`` (contract_bs_bs.jl:430-442) does; with two or more join
# axes whose value sets differ between the operands that merge can skip matched
# pairs, and this mode reproduces the reference's output there.
JOIN_ORDER = "sorted"


class join_order:
    """Context manager: ``with join_order("reference"): so.contract(...)``."""

    def __init__(self, mode: str):
        _assert(mode in ("sorted", "reference"), f"unknown join order {mode!r}")
        self.mode = mode

    def __enter__(self):
        global JOIN_ORDER
        self.prev, JOIN_ORDER = JOIN_ORDER, self.mode
        return self

    def __exit__(self, *exc):
        global JOIN_ORDER
        JOIN_ORDER = self.prev
        return False


def _cmp_join(akey, bkey, posA, posB) -> int:
    """``_cmp_join_tuple`` (contract_bs_bs.jl:430-442), with one correction
    unless ``JOIN_ORDER`` is "reference".

    The join axes are the last prefix axes of the permuted operands and keys
    are sorted column-major, so the last join axis is the most significant; the
    reference compares the first one first, and with two or more join axes
    whose value sets differ between the operands its merge skips matched pairs.
    Comparing from the last join axis down keeps the merge consistent with the
    sort; wherever the reference's merge finds every match the two agree."""
    pairs = list(zip(posA, posB))
    if JOIN_ORDER == "sorted":
        pairs.reverse()
    for pa, pb in pairs:
        av, bv = akey[pa - 1], bkey[pb - 1]
        if av < bv:
            return -1
        if av > bv:
            return 1
    return 0


def _slice_any_nonzero(vec: np.ndarray, off: int, length: int) -> bool:
    return bool(np.any(vec[off: off + length] != 0))


# ───────────────────────────── BS × BS kernels ────────────────────────────


def contract_prefix_outer_bb(C: BS, labelsC, A: BS, labelsA, B: BS, labelsB, rlab) -> BS:
    """``contract_prefix_outer_bb!`` (contract_bs_bs.jl:173-263)."""
    _assert(rlab not in labelsC)
    PA, PB, PC = A.P, B.P, C.P
    Adense, Bdense, Cdense = labelsA[PA:], labelsB[PB:], labelsC[PC:]
    _assert(not (set(Adense) & set(Bdense)), "outer kernel assumes disjoint dense labels")
    if list(Cdense) == list(Adense) + list(Bdense):
        order = 1
    elif list(Cdense) == list(Bdense) + list(Adense):
        order = 2
    else:
        raise OracleError("C dense must be [A_dense...,B_dense...] or [B_dense..., A_dense...]")
    _assert(C.blksize == A.blksize * B.blksize)
    _assert(labelsA.index(rlab) + 1 == PA and labelsB.index(rlab) + 1 == PB)
    C.clear()
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    src = []
    for lab in labelsC[:PC]:
        if lab in mapA:
            src.append(mapA[lab])
        else:
            _assert(lab in mapB, f"Label {lab} not found in A or B")
            src.append(-mapB[lab])
    iA, nA, iB, nB = 0, len(A.keys), 0, len(B.keys)
    while iA < nA and iB < nB:
        rvA, rvB = A.keys[iA][PA - 1], B.keys[iB][PB - 1]
        if rvA < rvB:
            while iA < nA and A.keys[iA][PA - 1] == rvA:
                iA += 1
            continue
        if rvB < rvA:
            while iB < nB and B.keys[iB][PB - 1] == rvB:
                iB += 1
            continue
        b_lo = iB
        while iB < nB and B.keys[iB][PB - 1] == rvA:
            iB += 1
        b_hi = iB
        while iA < nA and A.keys[iA][PA - 1] == rvA:
            akey = A.keys[iA]
            Avec = A.block(A.ids[iA])
            for iB2 in range(b_lo, b_hi):
                bkey = B.keys[iB2]
                Bvec = B.block(B.ids[iB2])
                ckey = tuple(akey[s - 1] if s > 0 else bkey[-s - 1] for s in src)
                cid = C.ensure_block(ckey)
                Cvec = C.block(cid)
                if order == 1:
                    _outer_add(Cvec, Avec, Bvec)
                else:
                    _outer_add(Cvec, Bvec, Avec)
            iA += 1
    return C


def contract_dense_bb(C: BS, labelsC, A: BS, labelsA, B: BS, labelsB, rlab) -> BS:
    """``contract_dense_bb!`` (contract_bs_bs.jl:288-423)."""
    _assert(rlab not in labelsC)
    PA, PB, PC = A.P, B.P, C.P
    axisAr, axisBr = labelsA.index(rlab) + 1, labelsB.index(rlab) + 1
    _assert(axisAr > PA and axisBr > PB)
    if axisAr != A.N:
        perm = _find_permutation_for_tensor(PA, A.N, axisAr)
        A, labelsA = bs_permutedims(A, perm), [labelsA[p - 1] for p in perm]
    if axisBr != B.N:
        perm = _find_permutation_for_tensor(PB, B.N, axisBr)
        B, labelsB = bs_permutedims(B, perm), [labelsB[p - 1] for p in perm]
    R = A.dims[-1]
    _assert(B.dims[-1] == R)
    chunkA, chunkB = A.blksize // R, B.blksize // R
    _assert(C.n2 == (A.n2 - 1) + (B.n2 - 1))
    _assert(C.blksize == chunkA * chunkB)
    Awo, Bwo, Cd = list(labelsA[PA:-1]), list(labelsB[PB:-1]), list(labelsC[PC:])
    if Cd == Awo + Bwo:
        order = "AB"
    elif Cd == Bwo + Awo:
        order = "BA"
    else:
        raise OracleError("C dense tail must be [A_dense..., B_dense...] or [B_dense..., A_dense...]")
    C.clear()
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    srcA, srcB = [0] * PC, [0] * PC
    for j, lab in enumerate(labelsC[:PC]):
        if lab in mapA:
            _assert(mapA[lab] <= PA)
            srcA[j] = mapA[lab]
        else:
            _assert(mapB[lab] <= PB)
            srcB[j] = mapB[lab]
    for akey, aid in zip(A.keys, A.ids):
        Af = A.block(aid)
        for bkey, bid in zip(B.keys, B.ids):
            Bf = B.block(bid)
            ckey = tuple(akey[srcA[j] - 1] if srcA[j] else bkey[srcB[j] - 1] for j in range(PC))
            Cmat = None
            for r in range(R):
                ao, bo = r * chunkA, r * chunkB
                if not _slice_any_nonzero(Af, ao, chunkA):
                    continue
                if not _slice_any_nonzero(Bf, bo, chunkB):
                    continue
                if Cmat is None:
                    cid = C.ensure_block(ckey)
                    Cvec = C.block(cid)
                    Cmat = _cmat(Cvec, chunkA, chunkB) if order == "AB" else _cmat(Cvec, chunkB, chunkA)
                As, Bs = Af[ao: ao + chunkA], Bf[bo: bo + chunkB]
                if order == "AB":
                    _rank1_add(Cmat, As, Bs)
                else:
                    _rank1_add(Cmat, Bs, As)
    return C


def contract_shared_bb(C: BS, labelsC, A: BS, labelsA, B: BS, labelsB, shared) -> BS:
    """``contract_shared!`` BS×BS (contract_bs_bs.jl:572-730)."""
    for lab in shared:
        _assert(lab not in labelsC, f"shared label {lab} must be reduced (must not appear in labelsC)")
    PA, PB, PC = A.P, B.P, C.P
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    shared_prefix, shared_dense = [], []
    for lab in shared:
        _assert(lab in mapA and lab in mapB)
        ap, bp = mapA[lab] <= PA, mapB[lab] <= PB
        if ap and bp:
            shared_prefix.append(lab)
        elif (not ap) and (not bp):
            shared_dense.append(lab)
        else:
            raise OracleError(f"shared label {lab} crosses prefix/dense; not supported")
    red = set(shared_dense)
    red_dense = [l for l in labelsA[PA:] if l in red]
    keepA0 = [l for l in labelsA[PA:] if l not in red]
    keepB0 = [l for l in labelsB[PB:] if l not in red]
    mode, dkA, dkB = _cdense_grouping_and_orders(labelsC[PC:], keepA0, keepB0)
    if mode == "interleaved":
        raise OracleError("Cdense interleaves A/B kept dims; would require permuting C (unsupported; sort/fallback)")
    _assert(len(dkA) == len(keepA0) and set(dkA) == set(keepA0))
    _assert(len(dkB) == len(keepB0) and set(dkB) == set(keepB0))
    permA = _find_perm_A_join_dense(labelsA, PA, shared_prefix, dkA, red_dense)
    permB = _find_perm_B_join_dense_redfirst(labelsB, PB, shared_prefix, red_dense, dkB)
    A = bs_permutedims(A, permA)
    B = bs_permutedims(B, permB)
    labelsA = [labelsA[p - 1] for p in permA]
    labelsB = [labelsB[p - 1] for p in permB]
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    nkA, nkB, nred = len(dkA), len(dkB), len(red_dense)
    dA, dB = A.dims[PA:], B.dims[PB:]
    M = 1 if nkA == 0 else _prod(dA[:nkA])
    K = 1 if nred == 0 else _prod(dA[nkA:])
    N = 1 if nkB == 0 else _prod(dB[nred:])
    if nred > 0:
        _assert(K == _prod(dB[:nred]), "Reduced dense extents mismatch between A and B")
    _assert(C.blksize == M * N, "C.blksize must equal M*N")
    src = []
    for lab in labelsC[:PC]:
        if lab in mapA and mapA[lab] <= PA:
            src.append(mapA[lab])
        elif lab in mapB and mapB[lab] <= PB:
            src.append(-mapB[lab])
        else:
            raise OracleError(f"C prefix label {lab} must come from A/B prefix")
    jA = [mapA[l] for l in shared_prefix]
    jB = [mapB[l] for l in shared_prefix]
    C.clear()
    iA, nA, iB, nB = 0, len(A.keys), 0, len(B.keys)
    while iA < nA and iB < nB:
        c = _cmp_join(A.keys[iA], B.keys[iB], jA, jB)
        if c < 0:
            iA = _advance_run(A.keys, iA, nA, jA)
            continue
        if c > 0:
            iB = _advance_run(B.keys, iB, nB, jB)
            continue
        iA2 = _advance_run(A.keys, iA, nA, jA)
        iB2 = _advance_run(B.keys, iB, nB, jB)
        for ii in range(iA, iA2):
            akey = A.keys[ii]
            Amat = _cmat(A.block(A.ids[ii]), M, K)
            for jj in range(iB, iB2):
                bkey = B.keys[jj]
                Bmat = _cmat(B.block(B.ids[jj]), K, N)
                ckey = tuple(akey[s - 1] if s > 0 else bkey[-s - 1] for s in src)
                cid = C.ensure_block(ckey)
                Cvec = C.block(cid)
                if mode == "AthenB":
                    Cm = _cmat(Cvec, M, N)
                    Cm += Amat @ Bmat
                else:
                    Cm = _cmat(Cvec, N, M)
                    Cm += Bmat.T @ Amat.T
        iA, iB = iA2, iB2
    return C


# ───────────────────────────── BS × Dense kernels ─────────────────────────


def _move_axis_to_last_perm(Nd: int, axisr: int) -> List[int]:
    return [d for d in range(1, Nd + 1) if d != axisr] + [axisr]


def contract_prefix_outer_bd(C: BS, labelsC, A: BS, labelsA, B: np.ndarray, labelsB, rlab) -> BS:
    """``contract_prefix_outer_bd!`` (contract_bs_dense.jl:34-204), Kahan sums."""
    _assert(rlab not in labelsC)
    PA, PC = A.P, C.P
    _assert(labelsA.index(rlab) + 1 <= PA)
    A, labelsA = _permute_r_to_last_prefix(A, list(labelsA), rlab)
    NB = B.ndim
    axisBr = list(labelsB).index(rlab) + 1
    R = B.shape[axisBr - 1]
    Br = B if axisBr == NB else dense_permutedims(B, _move_axis_to_last_perm(NB, axisBr))
    chunkB = Br.size // R
    Bmat = Br.reshape((chunkB, R), order="F")
    Adense = list(labelsA[PA:])
    Bwo = [l for l in labelsB if l != rlab]
    Cd = list(labelsC[PC:])
    if Cd == Adense + Bwo:
        order = "AB"
    elif Cd == Bwo + Adense:
        order = "BA"
    else:
        raise OracleError("C dense tail must be [A_dense..., B_wo_r...] or [B_wo_r..., A_dense...]")
    chunkA = A.blksize
    _assert(C.blksize == chunkA * chunkB)
    C.clear()
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    src = []
    for lab in labelsC[:PC]:
        _assert(lab in mapA, f"C prefix label {lab} not in A")
        ax = mapA[lab]
        _assert(ax <= PA and lab != rlab)
        src.append(ax)
    nA = len(A.keys)
    ckeys = [tuple(A.keys[i][s - 1] for s in src) for i in range(nA)]
    perm = _sortperm(ckeys, lambda k: k)  # lexicographic sortperm(ckeys) (:126)
    i = 0
    while i < nA:
        ckey = ckeys[perm[i]]
        cid = C.ensure_block(ckey)
        Cvec = C.block(cid)
        j = i + 1
        while j < nA and ckeys[perm[j]] == ckey:
            j += 1
        nb = j - i
        Am = np.empty((chunkA, nb))
        Bm = np.empty((chunkB, nb))
        for k in range(nb):
            iAk = perm[i + k]
            rv = A.keys[iAk][PA - 1]
            _assert(1 <= rv <= R)
            Am[:, k] = A.block(A.ids[iAk])
            Bm[:, k] = Bmat[:, rv - 1]
        if order == "AB":
            Cm = _cmat(Cvec, chunkA, chunkB)
            comp = np.zeros((chunkA, chunkB))
            for k in range(nb):
                y = np.multiply.outer(Am[:, k], Bm[:, k]) - comp
                t = Cm + y
                comp = (t - Cm) - y
                Cm[...] = t
        else:
            Cm = _cmat(Cvec, chunkB, chunkA)
            comp = np.zeros((chunkB, chunkA))
            for k in range(nb):
                y = np.multiply.outer(Bm[:, k], Am[:, k]) - comp
                t = Cm + y
                comp = (t - Cm) - y
                Cm[...] = t
        i = j
    return C


def contract_dense_bd(C: BS, labelsC, A: BS, labelsA, B: np.ndarray, labelsB, rlab) -> BS:
    """``contract_dense_bd!`` (contract_bs_dense.jl:248-392)."""
    _assert(rlab not in labelsC)
    PA, PC = A.P, C.P
    axisAr = labelsA.index(rlab) + 1
    axisBr = list(labelsB).index(rlab) + 1
    _assert(axisAr > PA)
    labelsA = list(labelsA)
    if axisAr != A.N:
        perm = _find_permutation_for_tensor(PA, A.N, axisAr)
        A, labelsA = bs_permutedims(A, perm), [labelsA[p - 1] for p in perm]
    NB = B.ndim
    labelsB = list(labelsB)
    Bp = B
    if axisBr != NB:
        permB = _move_axis_to_last_perm(NB, axisBr)
        Bp = dense_permutedims(B, permB)
        labelsB = [labelsB[p - 1] for p in permB]
    R = A.dims[-1]
    _assert(Bp.shape[-1] == R)
    chunkA = A.blksize // R
    chunkB = _prod(Bp.shape[:-1])
    _assert(C.n2 == (A.n2 - 1) + (NB - 1))
    _assert(C.blksize == chunkA * chunkB)
    Awo, Bwo, Cd = list(labelsA[PA:-1]), list(labelsB[:-1]), list(labelsC[PC:])
    if Cd == Awo + Bwo:
        order = "AB"
    elif Cd == Bwo + Awo:
        order = "BA"
    else:
        raise OracleError("C dense tail must be [A_dense..., B_dense...] or [B_dense..., A_dense...]")
    C.clear()
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    srcA = []
    for lab in labelsC[:PC]:
        _assert(mapA[lab] <= PA)
        srcA.append(mapA[lab])
    Bf = Bp.reshape(-1, order="F")
    for akey, aid in zip(A.keys, A.ids):
        Af = A.block(aid)
        ckey = tuple(akey[s - 1] for s in srcA)
        Cmat = None
        for r in range(R):
            ao, bo = r * chunkA, r * chunkB
            if not _slice_any_nonzero(Af, ao, chunkA):
                continue
            if not _slice_any_nonzero(Bf, bo, chunkB):
                continue
            if Cmat is None:
                cid = C.ensure_block(ckey)
                Cvec = C.block(cid)
                Cmat = _cmat(Cvec, chunkA, chunkB) if order == "AB" else _cmat(Cvec, chunkB, chunkA)
            As, Bs = Af[ao: ao + chunkA], Bf[bo: bo + chunkB]
            if order == "AB":
                _rank1_add(Cmat, As, Bs)
            else:
                _rank1_add(Cmat, Bs, As)
    return C


def contract_shared_bd(C: BS, labelsC, A: BS, labelsA, B: np.ndarray, labelsB, shared) -> BS:
    """``contract_shared!`` BS×Dense (contract_bs_dense.jl:411-619)."""
    for lab in shared:
        _assert(lab not in labelsC, f"shared label {lab} must be reduced (must not appear in labelsC)")
    PA, PC, NB = A.P, C.P, B.ndim
    labelsA, labelsB = list(labelsA), list(labelsB)
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    shared_prefix, shared_dense = [], []
    for lab in shared:
        _assert(lab in mapA and lab in mapB)
        (shared_prefix if mapA[lab] <= PA else shared_dense).append(lab)
    red = set(shared_dense)
    red_dense = [l for l in labelsA[PA:] if l in red]
    keepA0 = [l for l in labelsA[PA:] if l not in red]
    keepB0 = [l for l in labelsB if l not in set(shared)]
    mode, dkA, dkB = _cdense_grouping_and_orders(labelsC[PC:], keepA0, keepB0)
    if mode == "interleaved":
        raise OracleError("Cdense interleaves A/B kept dims; would require permuting C (unsupported; sort/fallback)")
    _assert(len(dkA) == len(keepA0) and set(dkA) == set(keepA0))
    _assert(len(dkB) == len(keepB0) and set(dkB) == set(keepB0))
    permA = _find_perm_A_join_dense(labelsA, PA, shared_prefix, dkA, red_dense)
    permB = [mapB[l] for l in shared_prefix] + [mapB[l] for l in red_dense] + [mapB[l] for l in dkB]
    _assert(len(permB) == NB)
    if permA != list(range(1, A.N + 1)):
        A = bs_permutedims(A, permA)
        labelsA = [labelsA[p - 1] for p in permA]
        mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    Bp = B if permB == list(range(1, NB + 1)) else dense_permutedims(B, permB)
    nkA, nkB, nred, nsp = len(dkA), len(dkB), len(red_dense), len(shared_prefix)
    dA = A.dims[PA:]
    dB = Bp.shape
    M = 1 if nkA == 0 else _prod(dA[:nkA])
    K = 1 if nred == 0 else _prod(dA[nkA:])
    N = 1 if nkB == 0 else _prod(dB[nsp + nred:])
    if nred > 0:
        _assert(K == _prod(dB[nsp: nsp + nred]), "Reduced dense extents mismatch between A and B")
    _assert(C.blksize == M * N, "C.blksize must equal M*N")
    csrc = []
    for lab in labelsC[:PC]:
        _assert(lab in mapA, f"C prefix label {lab} must exist in A")
        ap = mapA[lab]
        _assert(ap <= PA and lab not in set(shared_prefix))
        csrc.append(ap)
    jA = [mapA[l] for l in shared_prefix]
    C.clear()
    iA, nA = 0, len(A.keys)
    while iA < nA:
        iA2 = _advance_run(A.keys, iA, nA, jA)
        akey0 = A.keys[iA]
        if nsp == 0:
            Bsub = Bp
        else:
            Bsub = Bp[tuple(akey0[p - 1] - 1 for p in jA)]
        Bmat = np.asarray(Bsub).reshape((K, N), order="F")
        for ii in range(iA, iA2):
            akey = A.keys[ii]
            Amat = _cmat(A.block(A.ids[ii]), M, K)
            ckey = tuple(akey[s - 1] for s in csrc)
            cid = C.ensure_block(ckey)
            Cvec = C.block(cid)
            if mode == "AthenB":
                Cm = _cmat(Cvec, M, N)
                Cm += Amat @ Bmat
            else:
                Cm = _cmat(Cvec, N, M)
                Cm += Bmat.T @ Amat.T
        iA = iA2
    return C


# ───────────────────────────── COO kernels ────────────────────────────────


def _ensure_rlab_last_and_sorted(A: COO, labels, rlab):
    """``ensure_rlab_last_and_sorted`` (contract_coo.jl:48-82)."""
    labels = list(labels)
    if labels[-1] == rlab:
        return A, labels
    labels2 = [l for l in labels if l != rlab] + [rlab]
    pos = {l: i + 1 for i, l in enumerate(labels)}
    perm = [pos[l] for l in labels2]
    A2 = coo_permutedims(A, perm)
    A2.dirty = True
    coo_sort(A2)
    return A2, labels2


def contract_coo_coo(C: COO, labelsC, A: COO, labelsA, B: COO, labelsB, rlab) -> COO:
    """COO×COO→COO ``contract!`` (contract_coo.jl:93-170). Duplicates are kept."""
    A, labelsA = _ensure_rlab_last_and_sorted(A, labelsA, rlab)
    B, labelsB = _ensure_rlab_last_and_sorted(B, labelsB, rlab)
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    src = []
    for lab in labelsC:
        src.append((1, mapA[lab]) if lab in mapA else (2, mapB[lab]))
    C.keys, C.vals, C.dirty = [], [], True
    i, j, nA, nB = 0, 0, len(A.keys), len(B.keys)
    while i < nA and j < nB:
        ra, rb = A.keys[i][-1], B.keys[j][-1]
        if ra < rb:
            i += 1
        elif rb < ra:
            j += 1
        else:
            jlo = j
            while j < nB and B.keys[j][-1] == rb:
                j += 1
            while i < nA and A.keys[i][-1] == ra:
                ac, av = A.keys[i], A.vals[i]
                for jj in range(jlo, j):
                    bc, bv = B.keys[jj], B.vals[jj]
                    cc = tuple(ac[p - 1] if s == 1 else bc[p - 1] for s, p in src)
                    v = float(np.float64(av) * np.float64(bv))
                    if v != 0.0:  # _push_term! drops exact zeros (:84-91)
                        C.keys.append(cc)
                        C.vals.append(v)
                        C.dirty = True
                i += 1
    return C


def _aligned_A_to_Cprefix(A: COO, labelsA, labelsC, PC, rlab):
    """``aligned_A_to_Cprefix`` (contract_coo_dense.jl:4-18)."""
    desired = list(labelsC[:PC]) + [rlab]
    pos = {l: i + 1 for i, l in enumerate(labelsA)}
    perm = [pos[l] for l in desired]
    A2 = coo_permutedims(A, perm)
    coo_sort(A2)
    return A2, desired


def _coo_dense_prepare_B(B: np.ndarray, labelsB, labelsC, PC, rlab):
    desired = [l for l in labelsC[PC:] if l != rlab]
    labelsB = list(labelsB)
    NB = B.ndim
    perm = [labelsB.index(l) + 1 for l in desired] + [labelsB.index(rlab) + 1]
    _assert(len(perm) == NB)
    if perm != list(range(1, NB + 1)):
        B = dense_permutedims(B, perm)
        labelsB = [labelsB[p - 1] for p in perm]
    return B, labelsB


def contract_coo_dense(C: BS, labelsC, A: COO, labelsA, B: np.ndarray, labelsB, rlab) -> BS:
    """COO×Dense→BS ``contract!`` (contract_coo_dense.jl:48-125)."""
    PC = C.P
    A, labelsA = _aligned_A_to_Cprefix(A, labelsA, labelsC, PC, rlab)
    B, labelsB = _coo_dense_prepare_B(B, labelsB, labelsC, PC, rlab)
    _assert(labelsB[-1] == rlab and rlab not in labelsC)
    _assert(PC == len(labelsA) - 1, "PC mismatch")
    _assert(C.n2 == len(labelsB) - 1, "N2 mismatch")
    _assert(list(labelsC[:PC]) == labelsA[:-1])
    _assert(list(labelsC[PC:]) == labelsB[:-1])
    R = B.shape[-1]
    chunk = _prod(B.shape[:-1])
    _assert(C.blksize == chunk)
    C.clear()
    Bv = B.reshape(-1, order="F")
    for ac, av in zip(A.keys, A.vals):
        rv = ac[-1]
        if not (1 <= rv <= R):
            continue
        cid = C.ensure_block(tuple(ac[:PC]))
        Cv = C.block(cid)
        off = (rv - 1) * chunk
        Cv += np.float64(av) * Bv[off: off + chunk]  # _axpy_chunk! (:21-33)
    return C


def contract_coo_bs(C: BS, labelsC, A: COO, labelsA, B: BS, labelsB, rlab) -> BS:
    """COO×BS→BS dispatch (contract_coo_bs.jl:14-46)."""
    axisBr = list(labelsB).index(rlab) + 1
    if axisBr <= B.P:
        A, labelsA = _ensure_rlab_last_and_sorted(A, labelsA, rlab)
        B, labelsB = _permute_r_to_last_prefix(B, list(labelsB), rlab)
        return _coo_bs_prefix(C, labelsC, A, labelsA, B, labelsB, rlab)
    A, labelsA = _ensure_rlab_last_and_sorted(A, labelsA, rlab)
    return _coo_bs_dense_index(C, labelsC, A, labelsA, B, list(labelsB), rlab)


def _coo_bs_prefix(C: BS, labelsC, A: COO, labelsA, B: BS, labelsB, rlab) -> BS:
    """``contract_prefix!`` (contract_coo_bs.jl:51-124)."""
    PB, PC, NA = B.P, C.P, A.N
    _assert(PC == NA + PB - 2)
    C.clear()
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    aR, bR = mapA[rlab], mapB[rlab]
    iA, nA, iB, nB = 0, len(A.keys), 0, len(B.keys)
    while iA < nA and iB < nB:
        rA, rB = A.keys[iA][aR - 1], B.keys[iB][bR - 1]
        if rA < rB:
            while iA < nA and A.keys[iA][aR - 1] == rA:
                iA += 1
        elif rB < rA:
            while iB < nB and B.keys[iB][bR - 1] == rB:
                iB += 1
        else:
            rv = rA
            b_lo = iB
            while iB < nB and B.keys[iB][bR - 1] == rv:
                iB += 1
            b_hi = iB
            while iA < nA and A.keys[iA][aR - 1] == rv:
                ac, av = A.keys[iA], np.float64(A.vals[iA])
                for iB2 in range(b_lo, b_hi):
                    bk = B.keys[iB2]
                    ck = []
                    for lab in labelsC[:PC]:
                        if lab in mapA:
                            ck.append(ac[mapA[lab] - 1])
                        else:
                            _assert(mapB[lab] <= PB)
                            ck.append(bk[mapB[lab] - 1])
                    cid = C.ensure_block(tuple(ck))
                    Cv = C.block(cid)
                    Cv += av * B.block(B.ids[iB2])  # _scale_add_block! (:4-10)
                iA += 1
    return C


def _coo_bs_dense_index(C: BS, labelsC, A: COO, labelsA, B: BS, labelsB, rlab) -> BS:
    """``contract_dense_index!`` (contract_coo_bs.jl:140-241)."""
    _assert(rlab not in labelsC)
    PB, PC, NA = B.P, C.P, A.N
    _assert(C.n2 == B.n2 - 1)
    axisBr = labelsB.index(rlab) + 1
    _assert(axisBr > PB)
    redpos = axisBr - PB
    _assert(labelsA.index(rlab) + 1 == NA)
    ldense = list(labelsB[PB:])
    perm_dense = [d for d in range(1, B.n2 + 1) if d != redpos] + [redpos]
    Bp = B
    ldp = ldense
    if redpos != B.n2:
        Bp = bs_permutedims(B, list(range(1, PB + 1)) + [PB + d for d in perm_dense])
        ldp = [ldense[d - 1] for d in perm_dense]
    _assert(ldp[-1] == rlab)
    tdims = Bp.dims[PB:]
    dim_r = tdims[-1]
    chunk = _prod(tdims[:-1])
    _assert(list(labelsC[PC:]) == ldp[:-1])
    _assert(C.blksize == chunk)
    C.clear()
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    srcA, srcB = [0] * PC, [0] * PC
    for j, lab in enumerate(labelsC[:PC]):
        if lab in mapA:
            srcA[j] = mapA[lab]
        else:
            _assert(mapB[lab] <= PB)
            srcB[j] = mapB[lab]
    for ac, av in zip(A.keys, A.vals):
        rv = ac[NA - 1]
        _assert(1 <= rv <= dim_r)
        al = np.float64(av)
        for bk, bid in zip(Bp.keys, Bp.ids):
            ck = tuple(ac[srcA[j] - 1] if srcA[j] else bk[srcB[j] - 1] for j in range(PC))
            Bv = Bp.block(bid)
            off = (rv - 1) * chunk
            tmp = al * Bv[off: off + chunk]
            if not np.any(tmp != 0):
                continue
            cid = C.ensure_block(ck)
            C.block(cid)[...] += tmp
    return C


# ───────────────────────────── aliased kernels ────────────────────────────


class _AliasBook:
    """``_aliased_contribute!`` / ``_commit_aliased_dicts!`` (contract_aliased.jl:75-146).

    Julia ``Dict`` iteration order decides template ids of demoted blocks; the
    comparison unit is the per-key logical block, so insertion order is used.
    """

    def __init__(self, C: Aliased):
        self.C = C
        self.alias: Dict[Key, Tuple[int, float]] = {}
        self.accum: Dict[Key, np.ndarray] = {}
        self.tmpl: List[np.ndarray] = []

    def new_template(self, vec: np.ndarray) -> int:
        self.tmpl.append(vec)
        return len(self.tmpl)

    def contribute(self, ckey: Key, tid: int, scalar: float) -> None:
        scalar = np.float64(scalar)
        if ckey in self.accum:
            self.accum[ckey] = self.accum[ckey] + scalar * self.tmpl[tid - 1]
        elif ckey in self.alias:
            tprev, aprev = self.alias[ckey]
            if tprev == tid:
                self.alias[ckey] = (tprev, np.float64(aprev) + scalar)
            else:
                del self.alias[ckey]
                self.accum[ckey] = np.float64(aprev) * self.tmpl[tprev - 1] + scalar * self.tmpl[tid - 1]
        else:
            self.alias[ckey] = (tid, scalar)

    def commit(self) -> Aliased:
        C = self.C
        keys, aids, sc = [], [], []
        for k, (t, a) in self.alias.items():
            keys.append(k)
            aids.append(t)
            sc.append(float(a))
        for k, acc in self.accum.items():
            self.tmpl.append(acc)
            keys.append(k)
            aids.append(len(self.tmpl))
            sc.append(1.0)
        pd = C.dims[: C.P]
        p = _sortperm(keys, lambda k: prefix_lin(k, pd))
        C.keys = [keys[i] for i in p]
        C.alias_ids = [aids[i] for i in p]
        C.scalars = [sc[i] for i in p]
        C.templates = np.concatenate(self.tmpl) if self.tmpl else np.zeros(0)
        C.n_templates = len(self.tmpl)
        return C


def contract_aliased_coo_dense(C: Aliased, labelsC, A: COO, labelsA, B: np.ndarray, labelsB, rlab) -> Aliased:
    """COO×Dense→Aliased ``contract_aliased!`` (contract_aliased_coo_dense.jl:34-164)."""
    PC = C.P
    A, labelsA = _aligned_A_to_Cprefix(A, labelsA, labelsC, PC, rlab)
    B, labelsB = _coo_dense_prepare_B(B, labelsB, labelsC, PC, rlab)
    R = B.shape[-1]
    chunk = _prod(B.shape[:-1])
    _assert(C.blksize == chunk)
    Bv = B.reshape(-1, order="F")
    C.clear()
    book = _AliasBook(C)
    rv_to_tid: Dict[int, int] = {}
    for ac, av in zip(A.keys, A.vals):
        al = np.float64(av)
        rv = ac[-1]
        if not (1 <= rv <= R):
            continue
        ck = tuple(ac[:PC])
        off = (rv - 1) * chunk
        if ck in book.accum:
            book.accum[ck] = book.accum[ck] + al * Bv[off: off + chunk]
        elif ck in book.alias:
            tprev, aprev = book.alias.pop(ck)
            book.accum[ck] = np.float64(aprev) * book.tmpl[tprev - 1] + al * Bv[off: off + chunk]
        else:
            tid = rv_to_tid.get(rv, 0)
            if tid == 0:
                tid = book.new_template(Bv[off: off + chunk].copy())
                rv_to_tid[rv] = tid
            book.alias[ck] = (tid, al)
    return book.commit()


def _aliased_r_to_last_prefix(A: Aliased, labels, rlab):
    axisr = labels.index(rlab) + 1
    _assert(axisr <= A.P)
    if axisr == A.P:
        return A, list(labels)
    perm = [a for a in range(1, A.P + 1) if a != axisr] + [axisr] + list(range(A.P + 1, A.N + 1))
    return aliased_permutedims(A, perm), [labels[p - 1] for p in perm]


def _aliased_r_to_last_dense(A: Aliased, labels, rlab):
    axisr = labels.index(rlab) + 1
    _assert(axisr > A.P)
    if axisr == A.N:
        return A, list(labels)
    rl = axisr - A.P
    perm = list(range(1, A.P + 1)) + [A.P + d for d in range(1, A.n2 + 1) if d != rl] + [A.P + rl]
    return aliased_permutedims(A, perm), [labels[p - 1] for p in perm]


def contract_aliased_ad(C: Aliased, labelsC, A: Aliased, labelsA, B: np.ndarray, labelsB, rlab) -> Aliased:
    """Aliased×Dense single label (contract_aliased.jl:154-408)."""
    _assert(rlab not in labelsC)
    C.clear()
    labelsA, labelsB = list(labelsA), list(labelsB)
    if labelsA.index(rlab) + 1 <= A.P:
        A, labelsA = _aliased_r_to_last_prefix(A, labelsA, rlab)
        return _aliased_prefix_outer_ad(C, labelsC, A, labelsA, B, labelsB, rlab)
    A, labelsA = _aliased_r_to_last_dense(A, labelsA, rlab)
    return _aliased_dense_ad(C, labelsC, A, labelsA, B, labelsB, rlab)


def _bmat_r_last(B: np.ndarray, labelsB, rlab):
    NB = B.ndim
    ax = labelsB.index(rlab) + 1
    if ax != NB:
        perm = _move_axis_to_last_perm(NB, ax)
        B = dense_permutedims(B, perm)
        labelsB = [labelsB[p - 1] for p in perm]
    R = B.shape[-1]
    chunk = B.size // R
    return B.reshape((chunk, R), order="F"), labelsB, R, chunk


def _aliased_prefix_outer_ad(C, labelsC, A, labelsA, B, labelsB, rlab):
    """``_contract_aliased_prefix_outer_ad!`` (contract_aliased.jl:154-237)."""
    PA, PC = A.P, C.P
    Bm, labelsB, R, chunkB = _bmat_r_last(B, labelsB, rlab)
    _assert(C.blksize == A.blksize * chunkB)
    Ad, Bwo, Cd = list(labelsA[PA:]), list(labelsB[:-1]), list(labelsC[PC:])
    if Cd == Ad + Bwo:
        order = "AB"
    elif Cd == Bwo + Ad:
        order = "BA"
    else:
        raise OracleError("C dense tail must be [A_dense...,B_wo_r...] or [B_wo_r...,A_dense...]")
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    src = []
    for lab in labelsC[:PC]:
        ax = mapA[lab]
        _assert(ax <= PA and lab != rlab)
        src.append(ax)
    book = _AliasBook(C)
    ctm: Dict[Tuple[int, int], int] = {}
    for ak, tA, sA in zip(A.keys, A.alias_ids, A.scalars):
        rv = ak[PA - 1]
        if not (1 <= rv <= R):
            continue
        ck = tuple(ak[s - 1] for s in src)
        ct = ctm.get((tA, rv), 0)
        if ct == 0:
            nt = np.zeros(C.blksize)
            if order == "AB":
                _outer_add(nt, A.template(tA), Bm[:, rv - 1])
            else:
                _outer_add(nt, Bm[:, rv - 1], A.template(tA))
            ct = book.new_template(nt)
            ctm[(tA, rv)] = ct
        book.contribute(ck, ct, sA)
    return book.commit()


def _aliased_dense_ad(C, labelsC, A, labelsA, B, labelsB, rlab):
    """``_contract_aliased_dense_ad!`` (contract_aliased.jl:244-365)."""
    PA, PC = A.P, C.P
    _assert(PC == PA)
    Bm, labelsB, R, chunkB = _bmat_r_last(B, labelsB, rlab)
    _assert(A.dims[-1] == R)
    chunkA = A.blksize // R
    _assert(C.blksize == chunkA * chunkB)
    Awo, Bwo, Cd = list(labelsA[PA:-1]), list(labelsB[:-1]), list(labelsC[PC:])
    if Cd == Awo + Bwo:
        order = "AB"
    elif Cd == Bwo + Awo:
        order = "BA"
    else:
        raise OracleError("C dense tail must be [A_dense_wo_r...,B_wo_r...] or [B_wo_r...,A_dense_wo_r...]")
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    src = [mapA[l] for l in labelsC[:PC]]
    _assert(all(s <= PA for s in src))
    tmpl = []
    for t in range(1, A.n_templates + 1):
        Am = _cmat(A.template(t), chunkA, R)
        out = (Am @ Bm.T) if order == "AB" else (Bm @ Am.T)
        tmpl.append(np.asarray(out).reshape(-1, order="F"))
    keys = [tuple(k[s - 1] for s in src) for k in A.keys]
    pd = C.dims[:PC]
    p = _sortperm(keys, lambda k: prefix_lin(k, pd))
    C.keys = [keys[i] for i in p]
    C.alias_ids = [A.alias_ids[i] for i in p]
    C.scalars = [float(A.scalars[i]) for i in p]
    C.templates = np.concatenate(tmpl) if tmpl else np.zeros(0)
    C.n_templates = len(tmpl)
    return C


def contract_aliased_aa(C: Aliased, labelsC, A: Aliased, labelsA, B: Aliased, labelsB, rlab) -> Aliased:
    """Aliased×Aliased single label (contract_aliased.jl:417-690)."""
    _assert(rlab not in labelsC)
    C.clear()
    labelsA, labelsB = list(labelsA), list(labelsB)
    if labelsB.index(rlab) + 1 <= B.P:
        A, labelsA = _aliased_r_to_last_prefix(A, labelsA, rlab)
        B, labelsB = _aliased_r_to_last_prefix(B, labelsB, rlab)
        return _aliased_prefix_outer_aa(C, labelsC, A, labelsA, B, labelsB, rlab)
    _assert(labelsA.index(rlab) + 1 > A.P)
    A, labelsA = _aliased_r_to_last_dense(A, labelsA, rlab)
    B, labelsB = _aliased_r_to_last_dense(B, labelsB, rlab)
    return _aliased_dense_aa(C, labelsC, A, labelsA, B, labelsB, rlab)


def _aliased_prefix_outer_aa(C, labelsC, A, labelsA, B, labelsB, rlab):
    """``_contract_aliased_prefix_outer_aa!`` (contract_aliased.jl:417-520)."""
    PA, PB, PC = A.P, B.P, C.P
    _assert(C.blksize == A.blksize * B.blksize)
    Ad, Bd, Cd = list(labelsA[PA:]), list(labelsB[PB:]), list(labelsC[PC:])
    if Cd == Ad + Bd:
        order = 1
    elif Cd == Bd + Ad:
        order = 2
    else:
        raise OracleError("C dense must be [A_dense...,B_dense...] or [B_dense...,A_dense...]")
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    src = []
    for lab in labelsC[:PC]:
        if lab in mapA and mapA[lab] != mapA[rlab]:
            src.append(mapA[lab])
        else:
            _assert(lab in mapB and mapB[lab] <= PB and lab != rlab)
            src.append(-mapB[lab])
    book = _AliasBook(C)
    ctm: Dict[Tuple[int, int], int] = {}
    iA, nA, iB, nB = 0, len(A.keys), 0, len(B.keys)
    while iA < nA and iB < nB:
        rvA, rvB = A.keys[iA][PA - 1], B.keys[iB][PB - 1]
        if rvA < rvB:
            while iA < nA and A.keys[iA][PA - 1] == rvA:
                iA += 1
            continue
        if rvB < rvA:
            while iB < nB and B.keys[iB][PB - 1] == rvB:
                iB += 1
            continue
        b_lo = iB
        while iB < nB and B.keys[iB][PB - 1] == rvA:
            iB += 1
        b_hi = iB
        while iA < nA and A.keys[iA][PA - 1] == rvA:
            ak, tA, aA = A.keys[iA], A.alias_ids[iA], np.float64(A.scalars[iA])
            for j in range(b_lo, b_hi):
                bk, tB, aB = B.keys[j], B.alias_ids[j], np.float64(B.scalars[j])
                ct = ctm.get((tA, tB), 0)
                if ct == 0:
                    nt = np.zeros(C.blksize)
                    if order == 1:
                        _outer_add(nt, A.template(tA), B.template(tB))
                    else:
                        _outer_add(nt, B.template(tB), A.template(tA))
                    ct = book.new_template(nt)
                    ctm[(tA, tB)] = ct
                ck = tuple(ak[s - 1] if s > 0 else bk[-s - 1] for s in src)
                book.contribute(ck, ct, aA * aB)
            iA += 1
    return book.commit()


def _aliased_dense_aa(C, labelsC, A, labelsA, B, labelsB, rlab):
    """``_contract_aliased_dense_aa!`` (contract_aliased.jl:527-643)."""
    PA, PB, PC = A.P, B.P, C.P
    R = A.dims[-1]
    _assert(B.dims[-1] == R)
    chunkA, chunkB = A.blksize // R, B.blksize // R
    _assert(C.blksize == chunkA * chunkB)
    Awo, Bwo, Cd = list(labelsA[PA:-1]), list(labelsB[PB:-1]), list(labelsC[PC:])
    if Cd == Awo + Bwo:
        order = "AB"
    elif Cd == Bwo + Awo:
        order = "BA"
    else:
        raise OracleError("C dense tail must be [A_dense_wo_r...,B_dense_wo_r...] or swapped")
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    srcA, srcB = [0] * PC, [0] * PC
    for j, lab in enumerate(labelsC[:PC]):
        if lab in mapA:
            srcA[j] = mapA[lab]
        else:
            srcB[j] = mapB[lab]
    book = _AliasBook(C)
    ctm: Dict[Tuple[int, int], int] = {}
    for ak, tA, sA in zip(A.keys, A.alias_ids, A.scalars):
        for bk, tB, sB in zip(B.keys, B.alias_ids, B.scalars):
            ct = ctm.get((tA, tB), 0)
            if ct == 0:
                Am = _cmat(A.template(tA), chunkA, R)
                Bm = _cmat(B.template(tB), chunkB, R)
                out = (Am @ Bm.T) if order == "AB" else (Bm @ Am.T)
                ct = book.new_template(np.asarray(out).reshape(-1, order="F"))
                ctm[(tA, tB)] = ct
            ck = tuple(ak[srcA[j] - 1] if srcA[j] else bk[srcB[j] - 1] for j in range(PC))
            book.contribute(ck, ct, np.float64(sA) * np.float64(sB))
    return book.commit()


def contract_shared_aliased_ad(C: Aliased, labelsC, A: Aliased, labelsA, B: np.ndarray, labelsB, shared) -> Aliased:
    """``contract_shared!`` Aliased×Dense (contract_aliased_shared.jl:103-302)."""
    for lab in shared:
        _assert(lab not in labelsC)
    C.clear()
    PA, PC, NB = A.P, C.P, B.ndim
    labelsA, labelsB = list(labelsA), list(labelsB)
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    shared_prefix, shared_dense = [], []
    for lab in shared:
        _assert(lab in mapA and lab in mapB)
        (shared_prefix if mapA[lab] <= PA else shared_dense).append(lab)
    red = set(shared_dense)
    red_dense = [l for l in labelsA[PA:] if l in red]
    keepA0 = [l for l in labelsA[PA:] if l not in red]
    keepB0 = [l for l in labelsB if l not in set(shared)]
    mode, dkA, dkB = _cdense_grouping_and_orders(labelsC[PC:], keepA0, keepB0)
    if mode == "interleaved":
        raise OracleError("Cdense interleaves A/B kept dims; unsupported")
    permA = _find_perm_A_join_dense(labelsA, PA, shared_prefix, dkA, red_dense)
    if permA != list(range(1, A.N + 1)):
        A = aliased_permutedims(A, permA)
        labelsA = [labelsA[p - 1] for p in permA]
        mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    permB = [mapB[l] for l in shared_prefix] + [mapB[l] for l in red_dense] + [mapB[l] for l in dkB]
    _assert(len(permB) == NB)
    Bp = B if permB == list(range(1, NB + 1)) else dense_permutedims(B, permB)
    nsp, nred, nkA, nkB = len(shared_prefix), len(red_dense), len(dkA), len(dkB)
    dA, dB = A.dims[PA:], Bp.shape
    M = 1 if nkA == 0 else _prod(dA[:nkA])
    K = 1 if nred == 0 else _prod(dA[nkA:])
    N = 1 if nkB == 0 else _prod(dB[nsp + nred:])
    if nred > 0:
        _assert(K == _prod(dB[nsp: nsp + nred]))
    _assert(C.blksize == M * N)
    csrc = []
    for lab in labelsC[:PC]:
        ap = mapA[lab]
        _assert(ap <= PA and lab not in set(shared_prefix))
        csrc.append(ap)
    jA = [mapA[l] for l in shared_prefix]
    strides = []
    s = 1
    for t in range(nsp):
        strides.append(s)
        s *= dB[t]
    book = _AliasBook(C)
    ctm: Dict[Tuple[int, int], int] = {}
    iA, nA = 0, len(A.keys)
    while iA < nA:
        iA2 = _advance_run(A.keys, iA, nA, jA)
        a0 = A.keys[iA]
        sp_lin = 1 + sum((a0[jA[t] - 1] - 1) * strides[t] for t in range(nsp))
        Bsub = Bp if nsp == 0 else Bp[tuple(a0[p - 1] - 1 for p in jA)]
        Bm = np.asarray(Bsub).reshape((K, N), order="F")
        for ii in range(iA, iA2):
            ak, tA, sA = A.keys[ii], A.alias_ids[ii], A.scalars[ii]
            ct = ctm.get((tA, sp_lin), 0)
            if ct == 0:
                Am = _cmat(A.template(tA), M, K)
                out = (Am @ Bm) if mode == "AthenB" else (Bm.T @ Am.T)
                ct = book.new_template(np.asarray(out).reshape(-1, order="F"))
                ctm[(tA, sp_lin)] = ct
            book.contribute(tuple(ak[s - 1] for s in csrc), ct, sA)
        iA = iA2
    return book.commit()


def contract_shared_aliased_aa(C: Aliased, labelsC, A: Aliased, labelsA, B: Aliased, labelsB, shared) -> Aliased:
    """``contract_shared!`` Aliased×Aliased (contract_aliased_shared.jl:325-523)."""
    for lab in shared:
        _assert(lab not in labelsC)
    C.clear()
    PA, PB, PC = A.P, B.P, C.P
    labelsA, labelsB = list(labelsA), list(labelsB)
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    shared_prefix, shared_dense = [], []
    for lab in shared:
        ap, bp = mapA[lab] <= PA, mapB[lab] <= PB
        if ap and bp:
            shared_prefix.append(lab)
        elif (not ap) and (not bp):
            shared_dense.append(lab)
        else:
            raise OracleError(f"shared label {lab} crosses prefix/dense boundary; not supported")
    red = set(shared_dense)
    red_dense = [l for l in labelsA[PA:] if l in red]
    keepA0 = [l for l in labelsA[PA:] if l not in red]
    keepB0 = [l for l in labelsB[PB:] if l not in red]
    mode, dkA, dkB = _cdense_grouping_and_orders(labelsC[PC:], keepA0, keepB0)
    if mode == "interleaved":
        raise OracleError("Cdense interleaves A/B kept dims; unsupported")
    permA = _find_perm_A_join_dense(labelsA, PA, shared_prefix, dkA, red_dense)
    permB = _find_perm_B_join_dense_redfirst(labelsB, PB, shared_prefix, red_dense, dkB)
    A = aliased_permutedims(A, permA)
    B = aliased_permutedims(B, permB)
    labelsA = [labelsA[p - 1] for p in permA]
    labelsB = [labelsB[p - 1] for p in permB]
    mapA = {l: i + 1 for i, l in enumerate(labelsA)}
    mapB = {l: i + 1 for i, l in enumerate(labelsB)}
    nkA, nkB, nred = len(dkA), len(dkB), len(red_dense)
    dA, dB = A.dims[PA:], B.dims[PB:]
    M = 1 if nkA == 0 else _prod(dA[:nkA])
    K = 1 if nred == 0 else _prod(dA[nkA:])
    N = 1 if nkB == 0 else _prod(dB[nred:])
    _assert(C.blksize == M * N)
    src = []
    for lab in labelsC[:PC]:
        if lab in mapA and mapA[lab] <= PA:
            src.append(mapA[lab])
        elif lab in mapB and mapB[lab] <= PB:
            src.append(-mapB[lab])
        else:
            raise OracleError(f"C prefix label {lab} must come from A or B sparse prefix")
    jA = [mapA[l] for l in shared_prefix]
    jB = [mapB[l] for l in shared_prefix]
    book = _AliasBook(C)
    ctm: Dict[Tuple[int, int], int] = {}
    iA, nA, iB, nB = 0, len(A.keys), 0, len(B.keys)
    while iA < nA and iB < nB:
        c = _cmp_join(A.keys[iA], B.keys[iB], jA, jB)
        if c < 0:
            iA = _advance_run(A.keys, iA, nA, jA)
            continue
        if c > 0:
            iB = _advance_run(B.keys, iB, nB, jB)
            continue
        iA2 = _advance_run(A.keys, iA, nA, jA)
        iB2 = _advance_run(B.keys, iB, nB, jB)
        for ii in range(iA, iA2):
            ak, tA, aA = A.keys[ii], A.alias_ids[ii], np.float64(A.scalars[ii])
            for jj in range(iB, iB2):
                bk, tB, aB = B.keys[jj], B.alias_ids[jj], np.float64(B.scalars[jj])
                ct = ctm.get((tA, tB), 0)
                if ct == 0:
                    Am = _cmat(A.template(tA), M, K)
                    Bm = _cmat(B.template(tB), K, N)
                    out = (Am @ Bm) if mode == "AthenB" else (Bm.T @ Am.T)
                    ct = book.new_template(np.asarray(out).reshape(-1, order="F"))
                    ctm[(tA, tB)] = ct
                ck = tuple(ak[s - 1] if s > 0 else bk[-s - 1] for s in src)
                book.contribute(ck, ct, aA * aB)
        iA, iB = iA2, iB2
    return book.commit()


# ───────────────────────────── dispatch ───────────────────────────────────


def contract(C, labelsC, A, labelsA, B, labelsB):
    """``contract!(C, labelsC, A, labelsA, B, labelsB)`` (contract.jl:37-104)."""
    labelsA, labelsB, labelsC = list(labelsA), list(labelsB), list(labelsC)
    _assert(len(labelsA) == len(dims_of(A)), "labelsA length must match A rank")
    _assert(len(labelsB) == len(dims_of(B)), "labelsB length must match B rank")
    _assert(len(labelsC) == len(dims_of(C)), "labelsC length must match C rank")
    setB = set(labelsB)
    shared = [l for l in labelsA if l in setB]
    reduced = [l for l in shared if l not in set(labelsC)]
    if len(reduced) == 1:
        _assert(len(shared) == 1, f"Expected exactly 1 shared label; got {shared}")
        rlab = reduced[0]
        da = dims_of(A)[labelsA.index(rlab)]
        db = dims_of(B)[labelsB.index(rlab)]
        _assert(da == db, f"Dim mismatch on shared label {rlab}")
        return _contract_single(C, labelsC, A, labelsA, B, labelsB, rlab)
    return _contract_shared(C, labelsC, A, labelsA, B, labelsB, shared)


def _contract_single(C, labelsC, A, labelsA, B, labelsB, rlab):
    if isinstance(C, COO) and isinstance(A, COO) and isinstance(B, COO):
        return contract_coo_coo(C, labelsC, A, labelsA, B, labelsB, rlab)
    if isinstance(C, BS) and isinstance(A, BS) and isinstance(B, BS):
        if labelsB.index(rlab) + 1 <= B.P:
            A2, lA = _permute_r_to_last_prefix(A, labelsA, rlab)
            B2, lB = _permute_r_to_last_prefix(B, labelsB, rlab)
            return contract_prefix_outer_bb(C, labelsC, A2, lA, B2, lB, rlab)
        return contract_dense_bb(C, labelsC, A, labelsA, B, labelsB, rlab)
    if isinstance(C, BS) and isinstance(A, COO) and isinstance(B, BS):
        return contract_coo_bs(C, labelsC, A, labelsA, B, labelsB, rlab)
    if isinstance(C, BS) and isinstance(A, COO) and is_dense_array(B):
        return contract_coo_dense(C, labelsC, A, labelsA, B, labelsB, rlab)
    if isinstance(C, BS) and isinstance(A, BS) and is_dense_array(B):
        if labelsA.index(rlab) + 1 <= A.P:
            return contract_prefix_outer_bd(C, labelsC, A, labelsA, B, labelsB, rlab)
        return contract_dense_bd(C, labelsC, A, labelsA, B, labelsB, rlab)
    if isinstance(C, Aliased) and isinstance(A, Aliased) and is_dense_array(B):
        return contract_aliased_ad(C, labelsC, A, labelsA, B, labelsB, rlab)
    if isinstance(C, Aliased) and isinstance(A, Aliased) and isinstance(B, Aliased):
        return contract_aliased_aa(C, labelsC, A, labelsA, B, labelsB, rlab)
    if isinstance(C, Aliased) and isinstance(A, COO) and is_dense_array(B):
        return contract_aliased_coo_dense(C, labelsC, A, labelsA, B, labelsB, rlab)
    raise OracleError(f"MethodError: no contract! for C={type(C).__name__}, A={type(A).__name__}, B={type(B).__name__}")


def _contract_shared(C, labelsC, A, labelsA, B, labelsB, shared):
    if isinstance(C, BS) and isinstance(A, BS) and isinstance(B, BS):
        return contract_shared_bb(C, labelsC, A, labelsA, B, labelsB, shared)
    if isinstance(C, BS) and isinstance(A, BS) and is_dense_array(B):
        return contract_shared_bd(C, labelsC, A, labelsA, B, labelsB, shared)
    if isinstance(C, Aliased) and isinstance(A, Aliased) and is_dense_array(B):
        return contract_shared_aliased_ad(C, labelsC, A, labelsA, B, labelsB, shared)
    if isinstance(C, Aliased) and isinstance(A, Aliased) and isinstance(B, Aliased):
        return contract_shared_aliased_aa(C, labelsC, A, labelsA, B, labelsB, shared)
    raise OracleError(f"MethodError: no contract_shared! for C={type(C).__name__}, A={type(A).__name__}, B={type(B).__name__}")


def contract_bs_bs_to_dense(dimsC, labelsC, A: BS, labelsA, B: BS, labelsB) -> np.ndarray:
    """``contract_bs_bs_to_dense!`` (contract_bs_bs.jl:736-754): P_C = 0 sink."""
    NC = len(dimsC)
    Cbs = BS.empty(dimsC, NC) if NC > 0 else BS((), 0, [], [], np.zeros(0))
    contract(Cbs, labelsC, A, labelsA, B, labelsB)
    out = np.zeros(dimsC)
    if Cbs.keys:
        blk = Cbs.block(Cbs.ids[0])
        out = blk.reshape(dimsC, order="F").copy() if NC else np.array(blk[0])
    return out


# ── vector-space hooks used by Krylov solvers (src/tensor_wrappers.jl:793-923) ──

def bs_norm(A: BS) -> float:
    """``norm(w) = norm(w.blocksparse.data)`` (tensor_wrappers.jl:796)."""
    return float(np.linalg.norm(A.data))


def bs_scale(alpha: float, A: BS) -> BS:
    """``alpha * w``: same keys and ids, ``T(alpha) .* data`` (tensor_wrappers.jl:803-810)."""
    return BS(A.dims, A.n2, list(A.keys), list(A.ids), float(alpha) * A.data)


def bs_copy(A: BS) -> BS:
    """``copy(w)`` (tensor_wrappers.jl:816-822)."""
    return BS(A.dims, A.n2, list(A.keys), list(A.ids), A.data.copy())


def bs_add(A: BS, B: BS) -> BS:
    """``wA + wB`` (tensor_wrappers.jl:825-838): C = copy(A); for each B block,
    ``_ensure_block!`` in C (new blocks start at zero) and ``c[i] += b[i]``."""
    _assert(A.dims == B.dims and A.n2 == B.n2, "dims differ")
    Cb = bs_copy(A)
    for k, ib in zip(B.keys, B.ids):
        ic = Cb.ensure_block(k)
        blk = Cb.block(ic)
        blk += B.block(ib)
    return Cb


def bs_fill(A: BS, x: float) -> BS:
    """``fill!(storage.blocksparse.data, x)`` (tensor_wrappers.jl:848-851)."""
    for s in A._slots:
        s[:] = x
    return A


def map_values(op: str, r: np.ndarray, a: np.ndarray, alpha: float = 1.0, beta: float = 1.0) -> np.ndarray:
    """``_apply_elementwise!(f, R, A)`` (tensor_wrappers.jl:854-868): f over the
    stored values by position; lengths must agree.  ``op`` names the f."""
    if len(r) != len(a):
        raise ValueError("Mismatched sparsity patterns in _external_map!")
    if op == "axpy":
        return r + alpha * a
    if op == "axpby":
        return beta * r + alpha * a
    if op == "copy":
        return a.copy()
    if op == "mul":
        return r * a
    raise ValueError(op)


def bs_dot(A: BS, B: BS) -> float:
    """``dot(x, y) = (dag(x) * y)[]`` for real block-sparse tensors: the full
    contraction (contract_bs_bs_to_dense!, contract_bs_bs.jl:736-754, every
    label shared) = sum over keys present in both of the block dot products."""
    _assert(A.dims == B.dims and A.n2 == B.n2, "dims differ")
    bb = B.blocks_by_key()
    s = 0.0
    for k, ia in zip(A.keys, A.ids):
        if k in bb:
            s += float(np.dot(A.block(ia), bb[k]))
    return s


def aliased_norm(A: "Aliased") -> float:
    """``norm`` of an aliased tensor (tensor_wrappers_aliased.jl:524-536):
    sqrt(sum_i sum_j abs2(scalars[i] * templates[alias_ids[i]][j]))."""
    s = 0.0
    for i in range(len(A.keys)):
        t = A.template(A.alias_ids[i])
        s += float(np.sum((A.scalars[i] * t) ** 2))
    return float(np.sqrt(s))


# ── axis fusion (link fusion after MPO x MPO) ─────────────────────────────────

def fuse_two_axes(A: BS, ax1: int, ax2: int) -> BS:
    """``fuse_two_axes!`` (src/blocksparse/conversions.jl:228-314), axes 1-based.

    Prefix pair: fused key (k[a2]-1)*d[a1] + k[a1] at a1, a2 dropped, blocks and
    key order kept as in the reference (fuse_sparse_axes does not re-sort).
    Tail pair: move the later tail axis right after the earlier one (stable),
    then fold the two adjacent axes."""
    N, P = A.N, A.P
    if not (1 <= ax1 <= N and 1 <= ax2 <= N) or ax1 == ax2:
        raise ValueError("axes must be distinct and in 1:N")
    s1, s2 = ax1 <= P, ax2 <= P
    if s1 != s2:
        raise ValueError("Cannot fuse across sparse-head and dense-tail axes")
    a1, a2 = min(ax1, ax2), max(ax1, ax2)
    if s1:
        d1, d2 = A.dims[a1 - 1], A.dims[a2 - 1]
        nd = tuple(d1 * d2 if i == a1 else A.dims[i - 1] for i in range(1, N + 1) if i != a2)
        keys = []
        for k in A.keys:
            f = (k[a2 - 1] - 1) * d1 + k[a1 - 1]
            keys.append(tuple(f if j == a1 else k[j - 1] for j in range(1, P + 1) if j != a2))
        out = BS(nd, A.n2)
        out.keys, out.ids, out._slots = keys, list(A.ids), [s.copy() for s in A._slots]
        return out
    p1, p2 = a1 - P, a2 - P
    B = A
    if p2 != p1 + 1:
        pb = list(range(1, A.n2 + 1))
        x = pb.pop(p2 - 1)
        pb.insert(p1, x)
        B = bs_permutedims(A, list(range(1, P + 1)) + [P + q for q in pb])
    nd = tuple(B.dims[a1 - 1] * B.dims[a1] if i == a1 else B.dims[i - 1] for i in range(1, N + 1) if i != a1 + 1)
    out = BS(nd, A.n2 - 1)
    out.keys, out.ids, out._slots = list(B.keys), list(B.ids), [s.copy() for s in B._slots]
    return out


def fuse_axes_coo(A: "COO", ax1: int, ax2: int) -> "COO":
    """``fuse_axes_coo`` (src/coo/conversions.jl:174-222): adjacent axes, ax1
    kept as the fast index at ax1 - (ax2 < ax1); the result is sorted."""
    N = len(A.dims)
    if ax1 == ax2 or not (1 <= ax1 <= N and 1 <= ax2 <= N):
        raise ValueError("axes must be distinct and in 1:N")
    _assert(abs(ax1 - ax2) == 1, "Currently only adjacent axes can be fused")
    dkeep, ddrop = A.dims[ax1 - 1], A.dims[ax2 - 1]
    out_ax = ax1 - (1 if ax2 < ax1 else 0)
    old = lambda j: j if j < ax2 else j + 1  # noqa: E731
    nd = tuple(dkeep * ddrop if j == out_ax else A.dims[old(j) - 1] for j in range(1, N))
    keys = [tuple((c[ax2 - 1] - 1) * dkeep + c[ax1 - 1] if j == out_ax else c[old(j) - 1] for j in range(1, N))
            for c in A.keys]
    C = COO(nd, keys, list(A.vals), True)
    return coo_sort(C)
