"""Thin block GEMMs (K <= 16, one side <= 16) whose output blocks share blocks
of the long operand: the planner groups the output blocks that read the same
operand block and the kernels take the group's strips in turn (strip s of
every member, then strip s + 1).  Results must equal numpy and, bit for bit,
the tiled kernel (same pair order, same DMMA k-steps), for both thin
orientations and for the persistent and the one-CTA-per-strip thin kernels.
"""
import contextlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def _bs(sb, ctx, dense, n2):
    from oracle import sparse_oracle as so
    t = so.blocksparse_from_dense(dense, n2)
    return sb.NewBlockSparseSorted(t.dims, n2, t.keys, t.ids, t.data, ctx=ctx)


@pytest.mark.parametrize("long_rows", [True, False])
def test_shared_long_operand_chunks(sb, capfd, long_rows):
    rng = np.random.Generator(np.random.PCG64(21))
    M, K, N = 70000, 6, 5  # 547 strips per output block, three blocks per group
    Ad = rng.standard_normal((2, M, K))
    Bd = rng.standard_normal((3, N, K))
    lC = ["i", "j", "m", "n"] if long_rows else ["i", "j", "n", "m"]
    want = np.einsum("imk,jnk->ijmn", Ad, Bd)
    if not long_rows:
        want = want.transpose(0, 1, 3, 2)
    outs = []
    for kv in ({}, {"SPARSEB_GEMM_THIN": 1}, {"SPARSEB_GEMM_THIN": 0}):
        with _env(SPARSEB_TRACE=1, **kv):
            ctx = sb.Context(0)
        C = sb.NewBlockSparseSorted.empty(want.shape, 2, ctx=ctx)
        sb.contract_(C, lC, _bs(sb, ctx, Ad, 2), ["i", "m", "k"], _bs(sb, ctx, Bd, 2), ["j", "n", "k"])
        outs.append((sb.to_dense(C), capfd.readouterr().err))
    (p, tp), (o, to), (t, tt) = outs
    assert "thin persistent" in tp and "interleaved" in tp, tp
    assert "interleaved" in to and "persistent" not in to, to
    assert "gemm: tiled" in tt, tt
    assert np.linalg.norm(p - want) <= 1e-13 * np.linalg.norm(want)
    assert np.array_equal(p, t) and np.array_equal(o, t)


def test_unshared_blocks_keep_their_order(sb, capfd):
    """One output block per long-operand block: nothing to interleave."""
    rng = np.random.Generator(np.random.PCG64(22))
    Ad = rng.standard_normal((2, 40000, 6))
    Bd = rng.standard_normal((1, 5, 6))
    with _env(SPARSEB_TRACE=1):
        ctx = sb.Context(0)
    C = sb.NewBlockSparseSorted.empty((2, 1, 40000, 5), 2, ctx=ctx)
    sb.contract_(C, ["i", "j", "m", "n"], _bs(sb, ctx, Ad, 2), ["i", "m", "k"], _bs(sb, ctx, Bd, 2), ["j", "n", "k"])
    tr = capfd.readouterr().err
    assert "thin persistent" in tr and "interleaved" not in tr, tr
    want = np.einsum("imk,jnk->ijmn", Ad, Bd)
    assert np.linalg.norm(sb.to_dense(C) - want) <= 1e-13 * np.linalg.norm(want)
