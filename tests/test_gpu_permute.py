"""Block-sparse tail permutes (``permutedims``, storage.jl:188-264) on the
device against the oracle, bit-exact (keys, key order and every value), for
each kernel the permute stage picks:

* contiguous runs (output axis 0 has unit source stride; leading axes that
  are contiguous in both layouts merge into one run of >= 32 doubles);
* the narrow transpose (the output axes before the unit-stride one,
  flattened, span 2..32: every tile's output is one contiguous run), with and
  without batch axes and with a partial last tile;
* the 64 x 64 tiled transpose (partial tiles on both sides, batch axes, a
  row axis of one or two output axes);
* the general gather (everything else).

Prefix axes are permuted at the same time, so the blocks also move.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so

pytestmark = pytest.mark.gpu

CASES = [
    # (tail dims, tail perm (1-based within the tail), kernel)
    ((40, 3, 5), (1, 3, 2), "runs"),
    ((8, 6, 5), (1, 2, 3), "runs (merged axes)"),
    ((70, 14), (2, 1), "narrow"),
    ((70, 14, 3), (2, 1, 3), "narrow, batch"),
    ((65, 2), (2, 1), "narrow, dv = 2"),
    ((140, 5, 2), (2, 1, 3), "narrow, two tiles and a partial one"),
    ((100, 37, 3), (2, 3, 1), "tiled, partial tiles, batch"),
    ((50, 40), (2, 1), "tiled"),
    ((37, 3, 5, 2), (2, 3, 1, 4), "narrow, row axis of two output axes"),
    ((40, 7, 9), (2, 3, 1), "tiled, row axis of two output axes"),
    ((3, 4, 5), (2, 3, 1), "general"),
    ((8, 6, 5), (1, 3, 2), "general (short run)"),
]


@pytest.mark.parametrize("tail,tperm,kind", CASES, ids=[c[2] for c in CASES])
def test_tail_permute_matches_oracle(tail, tperm, kind):
    import sparsebackends_b200 as sb
    rng = np.random.Generator(np.random.PCG64(len(tail) * 100 + sum(tail)))
    pre = (3, 4)
    dims = pre + tail
    keys = sorted({(int(rng.integers(1, 4)), int(rng.integers(1, 5))) for _ in range(8)}, key=lambda k: k[::-1])
    blk = int(np.prod(tail))
    data = rng.standard_normal(len(keys) * blk)
    A = sb.NewBlockSparseSorted(dims, len(tail), keys, None, data)
    R = so.BS(dims, len(tail), keys, list(range(1, len(keys) + 1)), data)
    perm = [2, 1] + [2 + t for t in tperm]
    Ap, Rp = sb.permutedims(A, perm), so.bs_permutedims(R, perm)
    assert Ap.dims == tuple(dims[p - 1] for p in perm)
    assert Ap.keys == Rp.keys
    got, want = Ap.blocks_by_key(), Rp.blocks_by_key()
    for k in want:
        assert np.array_equal(np.ravel(got[k], order="F"), np.ravel(want[k], order="F")), (kind, k)


def test_dense_permutes_each_kernel():
    import sparsebackends_b200 as sb
    rng = np.random.Generator(np.random.PCG64(3))
    for shape, perm in (((40, 33, 17), (3, 1, 2)), ((64, 3, 20), (1, 3, 2)), ((130, 9), (2, 1)),
                        ((33, 70, 2), (2, 3, 1)), ((6, 7, 5), (3, 1, 2)), ((3, 4, 5), (2, 3, 1))):
        D = rng.standard_normal(shape)
        got = sb.to_dense(sb.permutedims(sb.DenseTensor(D), list(perm)))
        assert np.array_equal(got, np.transpose(D, [p - 1 for p in perm])), (shape, perm)


@pytest.mark.parametrize("tperm", [(1, 3, 2), (1, 2, 3), (2, 1, 3), (3, 2, 1)])
def test_ragged_tail_permutes(tperm):
    """Ragged blocks (each at its own extents): permuting then padding equals
    padding then permuting, bit for bit.  Tail orders that keep axis 0 run the
    per-block row copy; the others the per-block gather."""
    import sparsebackends_b200 as sb
    rng = np.random.Generator(np.random.PCG64(sum(tperm) * 7 + tperm[0]))
    dims = (3, 4, 37, 6, 5)
    keys = sorted({(int(rng.integers(1, 4)), int(rng.integers(1, 5))) for _ in range(7)}, key=lambda k: k[::-1])
    exts = [(int(rng.integers(1, 38)), int(rng.integers(1, 7)), int(rng.integers(1, 6))) for _ in keys]
    data = np.concatenate([rng.standard_normal(int(np.prod(e))) for e in exts])
    A = sb.NewBlockSparseSorted(dims, 3, keys, None, data, block_dims=exts)
    perm = [2, 1] + [2 + t for t in tperm]
    P = sb.permutedims(A, perm)
    assert P.is_ragged
    # block extents travel with their blocks (keys re-sorted by the prefix swap)
    ext_of = {(k[1], k[0]): tuple(e[t - 1] for t in tperm) for k, e in zip(keys, exts)}
    assert P.block_dims == [ext_of[k] for k in P.keys]
    got = sb.to_uniform(P)
    want = sb.permutedims(sb.to_uniform(A), perm)
    assert got.keys == want.keys
    assert np.array_equal(got.data, want.data)
