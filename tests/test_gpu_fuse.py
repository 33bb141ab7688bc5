"""GPU axis fusion and the sparse-MPO sandwich flow against the oracle.

* fuse_two_axes! (block-sparse): prefix pairs (adjacent and not) and tail
  pairs (adjacent and not, the latter through the tail permute) are bit-exact
  per key against the oracle; output keys are sorted column-major;
* fuse_axes_coo: both orientations, keys in sorted order and values exact;
* the sandwich_mpo flow of test_sparse_psi.jl:6-10 on one site: P (COO) x H
  (dense) -> block-sparse, then P (COO) x that -> block-sparse, then fusion of
  the left link pair, exact against the oracle and the dense einsum.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so

pytestmark = pytest.mark.gpu


def _sb():
    import sparsebackends_b200 as sb
    return sb


def _dev(sb, X, ctx):
    return sb.NewBlockSparseSorted(X.dims, X.n2, X.keys, X.ids, X.data, ctx=ctx)


def _same(dev, ref):
    got, want = dev.blocks_by_key(), ref.blocks_by_key()
    assert set(got) == set(want)
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    P = len(ref.dims) - ref.n2
    lins = [so.prefix_lin(k, ref.dims[:P]) for k in dev.keys]
    assert lins == sorted(lins)
    assert tuple(dev.dims) == tuple(ref.dims)


@pytest.mark.parametrize("axes", [(1, 2), (2, 1), (1, 3), (2, 3), (4, 5), (4, 6), (6, 4), (5, 6)])
def test_fuse_blocksparse(axes):
    sb = _sb()
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(sum(axes)))
    D = rng.standard_normal((3, 4, 2, 2, 3, 5)) * (rng.random((3, 4, 2, 1, 1, 1)) < 0.5)
    D[0, 0, 0] += 1
    A = so.blocksparse_from_dense(D, 3)
    ref = so.fuse_two_axes(A, *axes)
    got = sb.fuse_axes(_dev(sb, A, ctx), *axes)
    assert got.n2 == ref.n2
    _same(got, ref)


@pytest.mark.parametrize("axes", [(1, 2), (2, 1), (3, 2), (3, 4)])
def test_fuse_coo(axes):
    sb = _sb()
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(7 + axes[0]))
    D = rng.standard_normal((3, 4, 2, 5)) * (rng.random((3, 4, 2, 5)) < 0.2)
    A = so.coo_from_dense(D)
    ref = so.fuse_axes_coo(A, *axes)
    got = sb.fuse_axes(sb.COOTensor(A.dims, A.keys, A.vals, ctx=ctx), *axes)
    assert tuple(got.dims) == tuple(ref.dims)
    assert got.keys == ref.keys and got.vals == ref.vals and not got.dirty


def test_fuse_errors():
    sb = _sb()
    ctx = sb.Context(0)
    A = sb.blocksparse_from_dense(np.ones((2, 3, 4)), 1, ctx=ctx)
    with pytest.raises(sb.SparseBackendsError) as e:
        sb.fuse_axes(A, 1, 3)
    assert e.value.code == 1  # ArgumentError: across prefix and tail
    c = sb.coo_from_dense(np.eye(6).reshape(2, 3, 6), ctx=ctx)
    with pytest.raises(sb.SparseBackendsError) as e:
        sb.fuse_axes(c, 1, 3)
    assert e.value.code == 9  # AssertionError: not adjacent
    r = sb.NewBlockSparseSorted((2, 3, 4), 2, [(1,)], None, np.ones(4), ctx=ctx, block_dims=[(2, 2)])
    with pytest.raises(sb.SparseBackendsError) as e:
        sb.fuse_axes(r, 2, 3)
    assert e.value.code == 4  # ragged tail fusion unsupported


def test_sandwich_mpo_site_flow():
    sb = _sb()
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(42))
    Pd = rng.standard_normal((2, 2, 3, 3)) * (rng.random((2, 2, 3, 3)) < 0.3)
    P2d = rng.standard_normal((2, 2, 3, 3)) * (rng.random((2, 2, 3, 3)) < 0.3)
    Hd = rng.standard_normal((2, 2, 4, 4))
    l1 = (["x", "pl", "pr", "s", "hl", "hr"], ["x", "c", "pl", "pr"], ["c", "s", "hl", "hr"])
    l2 = (["y", "ql", "qr", "x", "pl", "pr", "hl", "hr"], ["s", "y", "ql", "qr"], l1[0])
    # oracle
    P, P2 = so.coo_from_dense(Pd), so.coo_from_dense(P2d)
    O1 = so.BS.empty((2, 3, 3, 2, 4, 4), 3)
    so.contract(O1, l1[0], P, l1[1], Hd, l1[2])
    O2 = so.BS.empty((2, 3, 3, 2, 3, 3, 4, 4), 2)
    so.contract(O2, l2[0], P2, l2[1], O1, l2[2])
    OF = so.fuse_two_axes(O2, 2, 5)
    # device
    dP = sb.COOTensor(P.dims, P.keys, P.vals, ctx=ctx)
    dP2 = sb.COOTensor(P2.dims, P2.keys, P2.vals, ctx=ctx)
    G1 = sb.NewBlockSparseSorted.empty((2, 3, 3, 2, 4, 4), 3, ctx=ctx)
    sb.contract_(G1, l1[0], dP, l1[1], Hd, l1[2])
    G2 = sb.NewBlockSparseSorted.empty((2, 3, 3, 2, 3, 3, 4, 4), 2, ctx=ctx)
    sb.contract_(G2, l2[0], dP2, l2[1], G1, l2[2])
    GF = sb.fuse_axes(G2, 2, 5)
    _same(G1, O1)
    _same(G2, O2)
    _same(GF, OF)
    want = np.einsum("syuv,xcab,cshr->yuvxabhr", P2d, Pd, Hd)
    assert np.allclose(sb.to_dense(G2), want, atol=1e-13)
