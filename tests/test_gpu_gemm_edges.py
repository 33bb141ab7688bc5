"""The tiled block GEMM with its edges cut off (64x64 tiles for the body,
64x32 / 64x48 tiles for column edges of width <= 32 / <= 48, 32x64 / 48x64
tiles for row edges, one launch) against numpy and against the single-shape
launch.

Every C element is summed over the same k-tiles in the same order whatever
tile covers it, so at equal split-K the two launches agree bit for bit.  The
cases cover the three operand layouts the contraction kernels launch
(contract_dense_bb!: X·Yᵀ; contract_shared!: X·Y and Xᵀ·Yᵀ), blocks that are
all edge (M or N <= 32), exact multiples of 64 and the split-K reduction.
"""
import contextlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (M, K, N) per block; K >= 1024 (133 x 1100 x 150, 45 x 1100 x 300) takes
# the long-K tile order; 100, 107, 40, 45 and 300 have 48-wide edges
SHAPES = [(133, 70, 411), (20, 40, 150), (96, 33, 18), (200, 300, 100), (64, 64, 64), (18, 2000, 411),
          (133, 1100, 150), (100, 70, 107), (96, 33, 40), (45, 1100, 300)]


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as sbmod
    return sbmod


@contextlib.contextmanager
def _env(**kv):
    old = {k: os.environ.get(k) for k in kv}
    os.environ.update({k: str(v) for k, v in kv.items()})
    try:
        yield
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _ctx(sb, **kv):
    with _env(SPARSEB_TRACE=1, **kv):
        return sb.Context(0)


def _bs(sb, ctx, dense, n2):
    from oracle import sparse_oracle as so
    t = so.blocksparse_from_dense(dense, n2)
    return sb.NewBlockSparseSorted(t.dims, n2, t.keys, t.ids, t.data, ctx=ctx)


def _case(pattern, M, K, N, rng):
    if pattern == "dense_bb":  # one shared label, k, in both dense tails
        Ad = rng.standard_normal((3, M, K))
        Bd = rng.standard_normal((2, N, K))
        want = np.einsum("imk,jnk->ijmn", Ad, Bd)
        return (Ad, ["i", "m", "k"], 2), (Bd, ["j", "n", "k"], 2), ["i", "j", "m", "n"], want
    if pattern == "shared_AB":
        Ad = rng.standard_normal((3, 2, M, K))
        Bd = rng.standard_normal((2, 2, K, N))
        want = np.einsum("iqmk,jqkn->ijmn", Ad, Bd)
        return (Ad, ["i", "q", "m", "k"], 2), (Bd, ["j", "q", "k", "n"], 2), ["i", "j", "m", "n"], want
    Ad = rng.standard_normal((3, 2, M, K))  # shared_BA: C tail [n, m] = (A·B)ᵀ per block
    Bd = rng.standard_normal((2, 2, K, N))
    want = np.einsum("iqmk,jqkn->ijnm", Ad, Bd)
    return (Ad, ["i", "q", "m", "k"], 2), (Bd, ["j", "q", "k", "n"], 2), ["i", "j", "n", "m"], want


def _expect_edges(Mc, Nc):
    """Whether the planner cuts the edges of uniform Mc x Nc C blocks: the
    FLOP-weighted tile choice is 64x64 and the cut saves >= 3% of the padded
    work."""
    if (Nc <= 32 and Mc >= 128) or (Mc <= 32 and Nc >= 128) or (Mc >= 1024 and Nc >= 512):
        return False
    up = lambda v, t: -(-v // t) * t
    body64 = lambda v: v - v % 64 if 0 < v % 64 <= 48 else v
    edge = lambda e: 32 if e <= 32 else 48
    mm, nm = body64(Mc), body64(Nc)
    w64 = up(Mc, 64) * up(Nc, 64)
    wseg = up(mm, 64) * up(nm, 64)
    if nm < Nc:
        wseg += up(Mc, 64) * up(Nc - nm, edge(Nc - nm))
    if mm < Mc and nm:
        wseg += up(Mc - mm, edge(Mc - mm)) * up(nm, 64)
    return wseg < 0.97 * w64


def _run(sb, ctx, A, B, lC, want_shape):
    (Ad, lA, nA), (Bd, lB, nB) = A, B
    C = sb.NewBlockSparseSorted.empty(want_shape, 2, ctx=ctx)
    sb.contract_(C, lC, _bs(sb, ctx, Ad, nA), lA, _bs(sb, ctx, Bd, nB), lB)
    return sb.to_dense(C)


@pytest.mark.parametrize("pattern", ["dense_bb", "shared_AB", "shared_BA"])
@pytest.mark.parametrize("splitk", [1, 3])
def test_edge_tiles_match_numpy_and_single_shape(sb, capfd, pattern, splitk):
    rng = np.random.Generator(np.random.PCG64(11))
    for M, K, N in SHAPES:
        A, B, lC, want = _case(pattern, M, K, N, rng)
        edges = _ctx(sb, SPARSEB_GEMM_SPLITK=splitk)
        got = _run(sb, edges, A, B, lC, want.shape)
        trace_edges = capfd.readouterr().err
        single = _ctx(sb, SPARSEB_GEMM_SPLITK=splitk, SPARSEB_GEMM_EDGES=0, SPARSEB_GEMM_TILE="64x64")
        ref = _run(sb, single, A, B, lC, want.shape)
        trace_single = capfd.readouterr().err
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= 1e-13, (pattern, M, K, N, err)
        assert np.array_equal(got, ref), (pattern, M, K, N)
        Mc, Nc = (N, M) if pattern == "shared_BA" else (M, N)
        assert ("gemm: edges" in trace_edges) == _expect_edges(Mc, Nc), (Mc, Nc, trace_edges)
        assert f"sk{splitk}" in trace_edges and "gemm: tiled 64x64" in trace_single


def test_edge_tiles_ragged_blocks(sb, capfd):
    """Ragged operands: every C block has its own extents, so one launch mixes
    blocks with and without edges (and blocks that are all edge)."""
    rng = np.random.Generator(np.random.PCG64(12))
    ms, ks, ns = [18, 133, 64, 96, 100], [40, 250], [411, 20, 70, 107]
    # A[(i, q) | m, k], B[(j, q) | k, n]: block (i, q) of A is ms[i] x ks[q],
    # block (j, q) of B is ks[q] x ns[j]; C[(i, j) | m, n] sums over q.
    Akeys = [(i + 1, q + 1) for q in range(2) for i in range(len(ms))]
    Bkeys = [(j + 1, q + 1) for q in range(2) for j in range(len(ns))]
    Ab = {k: rng.standard_normal((ms[k[0] - 1], ks[k[1] - 1])) for k in Akeys}
    Bb = {k: rng.standard_normal((ks[k[1] - 1], ns[k[0] - 1])) for k in Bkeys}

    def tensor(ctx, keys, blocks, dims):
        data = np.concatenate([blocks[k].reshape(-1, order="F") for k in keys])
        return sb.NewBlockSparseSorted(dims, 2, keys, None, data, ctx=ctx, block_dims=[blocks[k].shape for k in keys])

    outs = []
    for kv in ({}, {"SPARSEB_GEMM_EDGES": 0, "SPARSEB_GEMM_TILE": "64x64"}):
        ctx = _ctx(sb, SPARSEB_GEMM_SPLITK=1, **kv)
        A = tensor(ctx, Akeys, Ab, (len(ms), 2, max(ms), max(ks)))
        B = tensor(ctx, Bkeys, Bb, (len(ns), 2, max(ks), max(ns)))
        C = sb.NewBlockSparseSorted.empty((len(ms), len(ns), max(ms), max(ns)), 2, ctx=ctx)
        sb.contract_(C, ["i", "j", "m", "n"], A, ["i", "q", "m", "k"], B, ["j", "q", "k", "n"])
        outs.append((sb.to_dense(sb.to_uniform(C)), capfd.readouterr().err))
    (got, tr), (ref, _) = outs
    assert "gemm: edges" in tr
    assert np.array_equal(got, ref)
    for i in range(len(ms)):
        for j in range(len(ns)):
            want = sum(Ab[(i + 1, q + 1)] @ Bb[(j + 1, q + 1)] for q in range(2))
            blk = got[i, j, :ms[i], :ns[j]]
            assert np.linalg.norm(blk - want) <= 1e-13 * np.linalg.norm(want)
