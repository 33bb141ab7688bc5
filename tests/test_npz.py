"""``.npz`` interchange of the reference's storage fields.

CPU: write/read round trips of every kind through the host layer, with the
field names and integer/float types a Julia writer would produce, and the
format checks.  GPU: device tensor -> file -> device tensor is bit-exact
(keys, ids = 1:n, values; ragged extents), and a file written from the
oracle's storage (allocation-order ids) loads into the same tensor.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from sparsebackends_b200 import npz


def test_host_round_trip_blocksparse(tmp_path):
    rng = np.random.Generator(np.random.PCG64(0))
    D = rng.standard_normal((4, 3, 2, 5)) * (rng.random((4, 3, 1, 1)) < 0.5)
    D[0, 0] += 1
    A = so.blocksparse_from_dense(D, 2)
    p = str(tmp_path / "a.npz")
    npz.write_npz(p, "blocksparse", dims=A.dims, n2=A.n2, keys=A.keys, ids=A.ids, data=A.data)
    d = npz.read_npz(p)
    assert d["kind"] == "blocksparse" and d["dims"] == A.dims and d["n2"] == 2 and d["blksize"] == 10
    assert d["keys"] == A.keys and d["ids"] == A.ids and np.array_equal(d["data"], A.data)
    with np.load(p) as z:
        assert z["keys"].dtype == np.int64 and z["keys"].shape == (len(A.keys), 2)
        assert z["data"].dtype == np.float64


def test_host_round_trip_other_kinds(tmp_path):
    p = str(tmp_path / "c.npz")
    npz.write_npz(p, "coo", dims=(3, 4), keys=[(3, 1), (1, 2)], vals=[0.5, -2.0], dirty=True)
    d = npz.read_npz(p)
    assert d["keys"] == [(3, 1), (1, 2)] and d["vals"].tolist() == [0.5, -2.0] and d["dirty"]
    npz.write_npz(p, "aliased", dims=(2, 2, 3), n2=1, templates=np.arange(6.0), keys=[(1, 1), (2, 2)],
                  alias_ids=[2, 1], scalars=[1.5, -1.0])
    d = npz.read_npz(p)
    assert d["alias_ids"] == [2, 1] and np.array_equal(d["templates"], np.arange(6.0))
    x = np.arange(12.0).reshape(3, 4)
    npz.write_npz(p, "dense", dims=x.shape, data=x)
    d = npz.read_npz(p)
    assert np.array_equal(d["data"].reshape(d["dims"], order="F"), x)


def test_format_checks(tmp_path):
    p = str(tmp_path / "bad.npz")
    np.savez(p, format=np.array("other"), version=np.array(1), kind=np.array("dense"), dims=np.array([1]))
    with pytest.raises(ValueError):
        npz.read_npz(p)
    with pytest.raises(ValueError):
        npz.write_npz(p, "sparse", dims=(1,))


@pytest.mark.gpu
def test_device_round_trip_bit_exact(tmp_path):
    import sparsebackends_b200 as sb
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(1))
    D = rng.standard_normal((5, 4, 3, 2)) * (rng.random((5, 4, 1, 1)) < 0.4)
    D[1, 2] += 1
    A = so.blocksparse_from_dense(D, 2)
    # oracle storage with allocation-order ids, written as a Julia dump would be
    p = str(tmp_path / "o.npz")
    npz.write_npz(p, "blocksparse", dims=A.dims, n2=A.n2, keys=A.keys, ids=A.ids, data=A.data)
    t = npz.load(p, ctx)
    assert t.keys == A.keys and t.blocks_by_key().keys() == A.blocks_by_key().keys()
    for k, v in A.blocks_by_key().items():
        assert np.array_equal(t.blocks_by_key()[k], v)
    q = str(tmp_path / "d.npz")
    npz.save(q, t)
    t2 = npz.load(q, ctx)
    assert t2.keys == t.keys and t2.ids == list(range(1, len(t.keys) + 1))
    assert np.array_equal(t2.data, t.data)
    # ragged
    r = sb.NewBlockSparseSorted((3, 2, 4, 5), 2, [(1, 1), (3, 2)], None, np.arange(20.0 + 6), ctx=ctx,
                                block_dims=[(4, 5), (2, 3)])
    npz.save(q, r)
    r2 = npz.load(q, ctx)
    assert r2.is_ragged and r2.block_dims == r.block_dims and np.array_equal(r2.data, r.data)
    # COO, aliased, dense
    c = sb.COOTensor((3, 4), [(3, 1), (1, 2)], [0.5, -2.0], dirty=True, ctx=ctx)
    npz.save(q, c)
    c2 = npz.load(q, ctx)
    assert c2.keys == c.keys and c2.vals == c.vals and c2.dirty
    a = sb.AliasedBlockSparse((2, 2, 3), 1, np.arange(6.0), [(1, 1), (2, 2)], [2, 1], [1.5, -1.0], ctx=ctx)
    npz.save(q, a)
    a2 = npz.load(q, ctx)
    for k, v in a.logical_blocks().items():
        assert np.array_equal(a2.logical_blocks()[k], v)
    x = sb.DenseTensor(np.arange(12.0).reshape(3, 4), ctx)
    npz.save(q, x)
    assert np.array_equal(npz.load(q, ctx).to_numpy(), x.to_numpy())
