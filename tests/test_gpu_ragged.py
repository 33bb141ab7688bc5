"""Ragged (per-sector) block extents: the GPU result on unpadded blocks must
equal the reference format's result on the zero-padded blocks.

Pinned two ways: against the CPU oracle run on the padded (reference-format)
tensors, and against the library's own uniform path; same key lists, blocks
equal to the unpadded sub-blocks within 1e-12 relative Frobenius error.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _layout_small():
    from sparsebackends_b200 import qn
    # Two-site H_eff of a 16-site Heisenberg chain at chi=64 (config 1 shapes):
    # centre-bond profile {4,12,32,12,4}, MPO w=5 graded {-2:1, 0:3, +2:1}.
    left = qn.U1Link([-5, -3, -1, 1, 3, 5], [2, 8, 22, 22, 8, 2])
    right = qn.U1Link([-3, -1, 1, 3], [7, 25, 25, 7])
    mpo = qn.mpo_link({-2: 1, 0: 3, 2: 1})
    return qn.HeffLayout(left, right, mpo)


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("seed", [3, 4])
def test_ragged_heff_chain_matches_padded_oracle_and_uniform_gpu(seed):
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    lay = _layout_small()
    rng = np.random.Generator(np.random.PCG64(seed))
    rag, pad = {}, {}
    for name in ("psi", "L", "W1", "W2", "R"):
        keys, data, exts = qn.random_block_tensor(lay, name, rng, 0.5, ragged=True)
        rag[name] = sb.NewBlockSparseSorted(lay.dims[name], lay.n2[name], keys, None, data, block_dims=exts)
        pad[name] = (keys, qn.pad_ragged(lay, name, keys, data, exts))
    # GPU, ragged
    chain_r = qn.HeffChain(lay)
    out_r = chain_r.apply(rag["psi"], rag["L"], rag["W1"], rag["W2"], rag["R"])
    assert out_r.is_ragged
    got = sb.to_uniform(out_r)
    # GPU, uniform (reference format)
    uni = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d) for n, (k, d) in pad.items()}
    chain_u = qn.HeffChain(lay)
    out_u = chain_u.apply(uni["psi"], uni["L"], uni["W1"], uni["W2"], uni["R"])
    # oracle on the padded tensors
    t = {n: so.BS(lay.dims[n], lay.n2[n], k, list(range(1, len(k) + 1)), d) for n, (k, d) in pad.items()}
    lab = lay.labels
    for c, a, b in qn.HeffChain.STEPS:
        t[c] = so.contract(so.BS.empty(lay.dims[c], lay.n2[c]), lab[c], t[a], lab[a], t[b], lab[b])
    ref = t["T4"]
    assert got.keys == ref.keys == out_u.keys
    gb, ub, rb = got.blocks_by_key(), out_u.blocks_by_key(), ref.blocks_by_key()
    for k in rb:
        assert _rel(gb[k], rb[k]) <= RTOL
        assert _rel(ub[k], rb[k]) <= RTOL
    # the ragged blocks are exactly the unpadded sub-blocks of the result
    for k, e in zip(out_r.keys, out_r.block_dims):
        full = rb[k].reshape(lay.dims["T4"][4:], order="F")
        sub = out_r.blocks_by_key()[k].reshape(e, order="F")
        assert _rel(sub, full[tuple(slice(0, x) for x in e)]) <= RTOL
        mask = np.ones(full.shape, bool)
        mask[tuple(slice(0, x) for x in e)] = False
        assert np.all(full[mask] == 0)


def test_ragged_mixed_operands_and_permutes():
    import sparsebackends_b200 as sb
    rng = np.random.Generator(np.random.PCG64(9))
    # A[(i, q) | (m, k)] ragged x B[(q, j) | (k, n)] uniform, forcing a key reorder of B
    I, Q, J, M, K, N = 3, 4, 2, 9, 7, 5
    # the m extent is graded by i (a sector label), k is ungraded
    m_ext = {i: int(rng.integers(1, M + 1)) for i in range(1, I + 1)}
    ext = {(i, q): (m_ext[i], K) for i in range(1, I + 1) for q in range(1, Q + 1)}
    keys = [k for k in ext if rng.random() < 0.8]
    Ad = np.zeros((I, Q, M, K))
    parts = []
    for k in keys:
        e = ext[k]
        blk = rng.standard_normal(e)
        Ad[k[0] - 1, k[1] - 1, : e[0], : e[1]] = blk
        parts.append(blk.reshape(-1, order="F"))
    A_r = sb.NewBlockSparseSorted((I, Q, M, K), 2, keys, None, np.concatenate(parts),
                                  block_dims=[ext[k] for k in keys])
    Bd = rng.standard_normal((Q, J, K, N)) * (rng.random((Q, J, 1, 1)) < 0.8)
    B = so.blocksparse_from_dense(Bd, 2)
    Bg = sb.NewBlockSparseSorted(B.dims, 2, B.keys, B.ids, B.data)
    A = so.blocksparse_from_dense(Ad, 2)
    lA, lB, lC = ["i", "q", "m", "k"], ["q", "j", "k", "n"], ["i", "j", "m", "n"]
    ref = so.contract(so.BS.empty((I, J, M, N), 2), lC, A, lA, B, lB)
    C = sb.NewBlockSparseSorted.empty((I, J, M, N), 2)
    sb.contract_(C, lC, A_r, lA, Bg, lB)
    assert C.is_ragged
    U = sb.to_uniform(C)
    # zero blocks of A (all-zero rows in a ragged extent) may be absent from the
    # dense reference; compare against the oracle on the same key set
    assert U.keys == ref.keys
    ub, rb = U.blocks_by_key(), ref.blocks_by_key()
    for k in rb:
        assert _rel(ub[k], rb[k]) <= RTOL
    # ragged permute round trip
    Ap = sb.permutedims(A_r, [2, 1, 4, 3])
    assert np.array_equal(sb.to_dense(Ap), np.transpose(Ad, (1, 0, 3, 2)))
    # crop/pad adapters
    Au = sb.to_uniform(A_r)
    assert np.array_equal(sb.to_dense(Au), Ad)
    A_back = sb.to_ragged(Au, A_r.block_dims)
    assert np.array_equal(A_back.data, A_r.data)
    with pytest.raises(sb.SparseBackendsError):
        sb.to_ragged(Au, [(1, 1)] * len(A_r.keys), check_zero=True)


def test_ragged_inconsistent_output_extents_rejected():
    """Extents must follow the sector labels: two pairs feeding one output
    block with different extents is an error, not a silent truncation."""
    import sparsebackends_b200 as sb
    A_r = sb.NewBlockSparseSorted((2, 2, 4, 3), 2, [(1, 1), (1, 2)], None, np.ones(2 * 3 + 4 * 3),
                                  block_dims=[(2, 3), (4, 3)])
    B = sb.NewBlockSparseSorted((2, 2, 3, 5), 2, [(1, 1), (2, 1)], None, np.ones(2 * 15))
    C = sb.NewBlockSparseSorted.empty((2, 2, 4, 5), 2)
    with pytest.raises(sb.SparseBackendsError) as ei:
        sb.contract_(C, ["i", "j", "m", "n"], A_r, ["i", "q", "m", "k"], B, ["q", "j", "k", "n"])
    assert ei.value.status == "SB_ERR_DIM_MISMATCH"


def test_ragged_operand_rejected_where_unsupported():
    import sparsebackends_b200 as sb
    A_r = sb.NewBlockSparseSorted((3, 4, 5), 2, [(1,)], None, np.ones(6), block_dims=[(2, 3)])
    B = sb.DenseTensor(np.ones((5, 2)))
    C = sb.NewBlockSparseSorted.empty((3, 4, 2), 2)
    with pytest.raises(sb.SparseBackendsError) as ei:
        sb.contract_(C, ["p", "x", "y"], A_r, ["p", "x", "r"], B, ["r", "y"])
    assert ei.value.status == "SB_ERR_UNSUPPORTED_LAYOUT"
