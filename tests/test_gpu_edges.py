"""GPU edge cases against the oracle: empty operands, no matching keys, unit
extents, ragged unit blocks and launches with more than 65535 blocks.

The reference's kernels empty C first and create blocks only from matched
keys (e.g. ta/contract_bs_dense.jl:93,307,546), so an operand without blocks
or a contraction whose shared prefix values never meet gives an empty C with
the caller's dims.  Large block counts exercise the plan arrays and the launch
shapes (grid.y over 65535 items, one CTA per C block strip).
"""
import os

import numpy as np
import pytest

from oracle import sparse_oracle as so
from tests.test_gpu_parity import assert_bs_equal, lib_empty_like, lib_operand, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as sbmod
    return sbmod


def _run(sb, C0, lC, A, lA, B, lB):
    Cref = so.contract(C0, lC, A, lA, B, lB)
    Cg = lib_empty_like(sb, C0)
    sb.contract_(Cg, lC, lib_operand(sb, A), lA, lib_operand(sb, B), lB)
    return Cg, Cref


def test_empty_operands_every_family(sb):
    rng = np.random.Generator(np.random.PCG64(1))
    A4 = so.BS.empty((4, 3, 5, 6), 2)
    B4 = so.blocksparse_from_dense(rng.standard_normal((2, 3, 6, 7)), 2)
    lA, lB, lC = ["i", "q", "m", "k"], ["j", "q", "k", "n"], ["i", "j", "m", "n"]
    for X, Y in ((A4, B4), (so.blocksparse_from_dense(rng.standard_normal((4, 3, 5, 6)), 2),
                            so.BS.empty((2, 3, 6, 7), 2))):
        Cg, Cref = _run(sb, so.BS.empty((4, 2, 5, 7), 2), lC, X, lA, Y, lB)
        assert Cref.keys == [] and Cg.keys == [] and Cg.dims == (4, 2, 5, 7)
    # BS x dense (shared), empty A
    Cg, Cref = _run(sb, so.BS.empty((4, 3, 5, 7), 2), ["i", "q", "m", "n"], A4, lA,
                    rng.standard_normal((6, 7)), ["k", "n"])
    assert Cg.keys == Cref.keys == []
    # COO x dense, empty COO
    Ce = so.COO((3, 4, 5))
    Cg, Cref = _run(sb, so.BS.empty((3, 4, 7), 1), ["a", "b", "n"], Ce, ["a", "b", "r"],
                    rng.standard_normal((5, 7)), ["r", "n"])
    assert Cg.keys == Cref.keys == []
    # COO x COO, empty A
    Bc = so.coo_from_dense(rng.standard_normal((5, 7)) * (rng.random((5, 7)) < 0.5))
    Cref = so.contract(so.COO((3, 4, 7)), ["a", "b", "n"], Ce, ["a", "b", "r"], Bc, ["r", "n"])
    Cg = sb.COOTensor((3, 4, 7))
    sb.contract_(Cg, ["a", "b", "n"], lib_operand(sb, Ce), ["a", "b", "r"], lib_operand(sb, Bc), ["r", "n"])
    assert Cg.keys == Cref.keys == []
    # COO x BS, empty B
    Ac = so.coo_from_dense(rng.standard_normal((3, 5)) * (rng.random((3, 5)) < 0.6))
    Cg, Cref = _run(sb, so.BS.empty((3, 4, 6), 1), ["a", "x", "y"], Ac, ["a", "r"], so.BS.empty((5, 4, 6), 1),
                    ["r", "x", "y"])
    assert Cg.keys == Cref.keys == []


def test_no_matching_keys(sb):
    rng = np.random.Generator(np.random.PCG64(2))
    Ad = np.zeros((4, 3, 5, 6))
    Bd = np.zeros((2, 3, 6, 7))
    Ad[:, 0] = rng.standard_normal((4, 5, 6))   # A only at q = 1
    Bd[:, 2] = rng.standard_normal((2, 6, 7))   # B only at q = 3
    A, B = so.blocksparse_from_dense(Ad, 2), so.blocksparse_from_dense(Bd, 2)
    Cg, Cref = _run(sb, so.BS.empty((4, 2, 5, 7), 2), ["i", "j", "m", "n"], A, ["i", "q", "m", "k"], B,
                    ["j", "q", "k", "n"])
    assert Cg.keys == Cref.keys == []
    assert np.array_equal(sb.to_dense(Cg), np.zeros((4, 2, 5, 7)))


def test_unit_extents(sb):
    rng = np.random.Generator(np.random.PCG64(3))
    A = so.blocksparse_from_dense(rng.standard_normal((3, 2, 1, 1)), 2)
    B = so.blocksparse_from_dense(rng.standard_normal((4, 2, 1, 1)), 2)
    Cg, Cref = _run(sb, so.BS.empty((3, 4, 1, 1), 2), ["i", "j", "m", "n"], A, ["i", "q", "m", "k"], B,
                    ["j", "q", "k", "n"])
    assert_bs_equal(Cg, Cref)
    # ragged operand whose blocks are 1 x 1 inside 3 x 4 tails
    keys = [(1, 1), (2, 1), (3, 2)]
    r = sb.NewBlockSparseSorted((3, 2, 3, 4), 2, keys, None, np.array([2.0, -1.0, 0.5]),
                                block_dims=[(1, 1)] * 3)
    u = sb.to_uniform(r)
    assert u.keys == keys and np.count_nonzero(u.data) == 3
    assert abs(sb.norm(r) - np.sqrt(4 + 1 + 0.25)) < 1e-15


@pytest.mark.parametrize("thin", ["auto", "0", "1"])
def test_more_than_65535_blocks(sb, thin):
    """90000 output blocks (300 x 300 prefix pairs), 2 x 2 tails: the
    persistent thin kernel in the automatic choice, the tiled kernel with
    SPARSEB_GEMM_THIN=0, the one-CTA-per-strip thin kernel with =1."""
    rng = np.random.Generator(np.random.PCG64(4))
    n = 300
    A = so.blocksparse_from_dense(rng.standard_normal((n, 1, 2, 2)), 2)
    B = so.blocksparse_from_dense(rng.standard_normal((n, 1, 2, 2)), 2)
    old = os.environ.get("SPARSEB_GEMM_THIN")
    if thin != "auto":
        os.environ["SPARSEB_GEMM_THIN"] = thin
    try:
        ctx = sb.Context(0)
    finally:
        if old is None:
            os.environ.pop("SPARSEB_GEMM_THIN", None)
        else:
            os.environ["SPARSEB_GEMM_THIN"] = old
    lC, lA, lB = ["i", "j", "m", "n"], ["i", "q", "m", "k"], ["j", "q", "k", "n"]
    Cg = sb.NewBlockSparseSorted.empty((n, n, 2, 2), 2, ctx=ctx)
    sb.contract_(Cg, lC, sb.NewBlockSparseSorted(A.dims, 2, A.keys, A.ids, A.data, ctx=ctx), lA,
                 sb.NewBlockSparseSorted(B.dims, 2, B.keys, B.ids, B.data, ctx=ctx), lB)
    Ad = so.bs_to_dense(A)[:, 0]
    Bd = so.bs_to_dense(B)[:, 0]
    want = np.einsum("imk,jkn->ijmn", Ad, Bd)
    got = sb.to_dense(Cg)
    assert len(Cg.keys) == n * n
    assert rel_err(got, want) <= 1e-13
    # vector ops over the same many-block tensor
    assert abs(sb.norm(Cg) - np.linalg.norm(want)) <= 1e-13 * np.linalg.norm(want)
    assert abs(sb.dot(Cg, Cg) - float(np.sum(want * want))) <= 1e-12 * float(np.sum(want * want))


def test_vector_ops_on_empty(sb):
    e = sb.NewBlockSparseSorted.empty((3, 4, 2), 1)
    assert sb.norm(e) == 0.0 and sb.dot(e, e) == 0.0
    s = sb.add(e, e)
    assert s.keys == [] and sb.copy(e).keys == [] and sb.similar(e).keys == []
    sb.scale_(e, 2.0)
    sb.fill_(e, 1.0)
    assert e.keys == []


def test_two_label_join_with_unequal_tuple_sets(sb):
    """Two shared prefix labels whose (w, s) value sets differ between A and B:
    every matched pair contributes (the merge compares in key-sort order)."""
    rng = np.random.Generator(np.random.PCG64(3))
    Ad = np.zeros((2, 3, 2, 4))
    Ad[:, 1] = rng.standard_normal((2, 2, 4))
    Bd = rng.standard_normal((3, 2, 3, 5))
    A, B = so.blocksparse_from_dense(Ad, 1), so.blocksparse_from_dense(Bd, 1)
    Cg, Cref = _run(sb, so.BS.empty((2, 3, 4, 5), 2), ["p", "t", "m", "n"], A, ["p", "w", "s", "m"], B,
                    ["w", "s", "t", "n"])
    assert_bs_equal(Cg, Cref)
    assert rel_err(sb.to_dense(Cg), np.einsum("pwsm,wstn->ptmn", Ad, Bd)) <= 1e-13
