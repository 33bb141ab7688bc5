"""GPU parity of the vector-space hooks and the device Lanczos eigensolver.

Vector hooks (src/tensor_wrappers.jl:793-923) against the oracle's
restatements, through the C ABI:
* x + y (key union), alpha*x, copy, similar, fill!, map! (axpy / axpby / copy /
  multiply) are exactly rounded elementwise operations: bit-exact;
* norm and dot are reductions in a different (fixed) order: 1e-14 relative;
* ragged and uniform layouts, dense and aliased tensors, and the error
  statuses of mismatched operands.

Lanczos (KrylovKit eigsolve restated in sparsebackends_b200.krylov) on a
Hermitian two-site H_eff: the device solver against the numpy oracle solver on
the same start vector (krylovdim 3, maxiter 1: the reference's DMRG setting;
Ritz value 1e-10 relative, Ritz vector 1e-8), and a converged solve against
exact diagonalisation of the dense H_eff (1e-9 relative).
"""
import numpy as np
import pytest

from oracle import krylov_oracle as ko
from oracle import sparse_oracle as so
from tests.heff_dense import heff_restricted, small_layout

pytestmark = pytest.mark.gpu


def _sb():
    import sparsebackends_b200 as sb
    return sb


def _pair(seed, dims=(5, 3, 6, 4), n2=2, pa=0.6, pb=0.6):
    rng = np.random.Generator(np.random.PCG64(seed))
    P = len(dims) - n2
    mask_shape = dims[:P] + (1,) * n2
    Ad = rng.standard_normal(dims) * (rng.random(mask_shape) < pa)
    Bd = rng.standard_normal(dims) * (rng.random(mask_shape) < pb)
    return Ad, Bd, so.blocksparse_from_dense(Ad, n2), so.blocksparse_from_dense(Bd, n2)


def _dev(sb, X, ctx):
    return sb.NewBlockSparseSorted(X.dims, X.n2, X.keys, X.ids, X.data, ctx=ctx)


def _same_blocks(dev, ref: so.BS):
    got = dev.blocks_by_key()
    want = ref.blocks_by_key()
    assert list(got) == sorted(want, key=lambda k: so.prefix_lin(k, ref.dims[: ref.P]))
    for k in want:
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_norm_dot_add_scale_match_oracle(seed):
    sb = _sb()
    ctx = sb.Context(0)
    Ad, Bd, A, B = _pair(seed)
    a, b = _dev(sb, A, ctx), _dev(sb, B, ctx)
    assert abs(sb.norm(a) - so.bs_norm(A)) <= 1e-14 * so.bs_norm(A)
    ref = so.bs_dot(A, B)
    assert abs(sb.dot(a, b) - ref) <= 1e-14 * max(1.0, np.linalg.norm(Ad) * np.linalg.norm(Bd))
    _same_blocks(sb.add(a, b), so.bs_add(A, B))
    _same_blocks(a + b, so.bs_add(A, B))
    _same_blocks(-1.75 * a, so.bs_scale(-1.75, A))
    _same_blocks(a / 4.0, so.bs_scale(0.25, A))
    _same_blocks(a - b, so.bs_add(A, so.bs_scale(-1.0, B)))


def test_copy_similar_fill_are_independent():
    sb = _sb()
    ctx = sb.Context(0)
    _, _, A, _ = _pair(3)
    a = _dev(sb, A, ctx)
    c = sb.copy(a)
    z = sb.similar(a)
    sb.fill_(a, 2.5)
    _same_blocks(c, A)
    assert z.keys == c.keys and not np.any(z.data)
    assert np.all(a.data == 2.5) and a.keys == c.keys


@pytest.mark.parametrize("op,alpha,beta", [("axpy", 0.37, 1.0), ("axpby", -1.3, 0.7), ("copy", 1.0, 1.0),
                                           ("mul", 1.0, 1.0)])
def test_map_ops_bit_exact(op, alpha, beta):
    sb = _sb()
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(4))
    keys = [(1, 1), (2, 1), (1, 3)]
    r0, a0 = rng.standard_normal(3 * 20), rng.standard_normal(3 * 20)
    R = sb.NewBlockSparseSorted((2, 3, 4, 5), 2, keys, None, r0, ctx=ctx)
    A = sb.NewBlockSparseSorted((2, 3, 4, 5), 2, keys, None, a0, ctx=ctx)
    codes = {"axpy": sb.MAP_AXPY, "axpby": sb.MAP_AXPBY, "copy": sb.MAP_COPY, "mul": sb.MAP_MUL}
    sb.map_(R, A, codes[op], alpha, beta)
    # device payload is in sorted-key order; build the oracle arrays the same way
    order = np.argsort([so.prefix_lin(k, (2, 3)) for k in keys], kind="stable")
    rs = np.concatenate([r0[i * 20:(i + 1) * 20] for i in order])
    as_ = np.concatenate([a0[i * 20:(i + 1) * 20] for i in order])
    assert np.array_equal(R.data, so.map_values(op, rs, as_, alpha, beta))


def test_dense_and_ragged_vectors():
    sb = _sb()
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(5))
    x, y = rng.standard_normal((7, 9)), rng.standard_normal((7, 9))
    dx, dy = sb.DenseTensor(x, ctx), sb.DenseTensor(y, ctx)
    assert abs(sb.dot(dx, dy) - float(np.sum(x * y))) < 1e-13
    assert abs(sb.norm(dx) - np.linalg.norm(x)) < 1e-13
    assert np.array_equal(sb.add(dx, dy).to_numpy(), x + y)
    # ragged: block extents per key; dot/add against the zero-padded uniform copy
    dims, keys = (3, 2, 4, 5), [(1, 1), (3, 1), (2, 2)]
    ext = [(4, 5), (2, 3), (1, 5)]
    d1 = np.concatenate([rng.standard_normal(int(np.prod(e))) for e in ext])
    d2 = np.concatenate([rng.standard_normal(int(np.prod(e))) for e in ext])
    r1 = sb.NewBlockSparseSorted(dims, 2, keys, None, d1, ctx=ctx, block_dims=ext)
    r2 = sb.NewBlockSparseSorted(dims, 2, keys[:2], None, d2[:26], ctx=ctx, block_dims=ext[:2])
    u1, u2 = sb.to_uniform(r1), sb.to_uniform(r2)
    assert abs(sb.dot(r1, r2) - sb.dot(u1, u2)) < 1e-13
    assert abs(sb.norm(r1) - np.linalg.norm(d1)) < 1e-13
    s = sb.add(r1, r2)
    assert s.is_ragged and s.block_dims == r1.block_dims
    assert np.array_equal(sb.to_uniform(s).data, sb.add(u1, u2).data)


def test_aliased_norm_and_scalar_map():
    sb = _sb()
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(6))
    tmpl = rng.standard_normal(2 * 6)
    keys, alias, scal = [(1, 1), (2, 1), (2, 2)], [1, 2, 1], [0.5, -2.0, 3.0]
    A = sb.AliasedBlockSparse((2, 2, 2, 3), 2, tmpl, keys, alias, scal, ctx=ctx)
    ref = so.Aliased((2, 2, 2, 3), 2, tmpl.copy(), 2, list(keys), list(alias), list(scal))
    assert abs(sb.norm(A) - so.aliased_norm(ref)) < 1e-13
    B = sb.copy(A)
    sb.map_(A, B, sb.MAP_AXPY, 2.0)  # scalars: s + 2 s = 3 s
    lb = A.logical_blocks()
    for k, s, t in zip(keys, scal, alias):
        assert np.array_equal(lb[k], (s + 2.0 * s) * tmpl[(t - 1) * 6: t * 6])


def test_vector_op_errors():
    sb = _sb()
    ctx = sb.Context(0)
    _, _, A, B = _pair(7, pa=0.9, pb=0.3)
    a, b = _dev(sb, A, ctx), _dev(sb, B, ctx)
    if len(A.keys) != len(B.keys):
        with pytest.raises(sb.SparseBackendsError) as e:
            sb.map_(a, b, sb.MAP_AXPY, 1.0)
        assert e.value.code == 2  # SB_ERR_DIM_MISMATCH: mismatched sparsity patterns
    c = sb.NewBlockSparseSorted((5, 3, 6, 5), 2, [(1, 1)], None, np.ones(30), ctx=ctx)
    with pytest.raises(sb.SparseBackendsError) as e:
        sb.dot(a, c)
    assert e.value.code == 2
    coo = sb.coo_from_dense(np.eye(3), ctx=ctx)
    with pytest.raises(sb.SparseBackendsError) as e:
        sb.dot(coo, coo)
    assert e.value.code == 5  # SB_ERR_UNSUPPORTED_TYPES


# ── Lanczos ────────────────────────────────────────────────────────────────

def _heff_problem(seed, chi=24):
    sb = _sb()
    from sparsebackends_b200 import qn
    lay = small_layout(chi)
    rng = np.random.Generator(np.random.PCG64(seed))
    ops = qn.hermitian_operators(lay, rng)
    pk, pd, pe = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    ctx = sb.Context(0)
    dev = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx, block_dims=e)
           for n, (k, d, e) in ops.items()}
    psi = sb.NewBlockSparseSorted(lay.dims["psi"], 2, pk, None, pd, ctx=ctx, block_dims=pe)
    op = qn.HeffOperator(lay, dev["L"], dev["W1"], dev["W2"], dev["R"], ctx)
    H = heff_restricted(lay, ops, pk, pe)
    return sb, lay, op, psi, pd, H


def _close_up_to_sign(x, y, tol):
    return min(np.linalg.norm(x - y), np.linalg.norm(x + y)) <= tol * np.linalg.norm(y)


@pytest.mark.parametrize("seed", [21, 22])
def test_lanczos_krylovdim3_matches_oracle(seed):
    from sparsebackends_b200 import krylov
    sb, lay, op, psi, pd, H = _heff_problem(seed)
    vals, vecs, info = krylov.eigsolve(op, psi, 1, "SR", krylovdim=3, maxiter=1, tol=1e-14)
    rv, rvec, conv, nit, nops = ko.lanczos_eigsolve(lambda v: H @ v, pd, 1, "SR", krylovdim=3, maxiter=1, tol=1e-14)
    assert (info.numiter, info.numops) == (nit, nops) == (1, 3)
    assert op.calls == 3
    assert abs(vals[0] - rv[0]) <= 1e-10 * abs(rv[0])
    assert _close_up_to_sign(vecs[0].data, rvec[0], 1e-8)
    # the matvec through the device chain equals the dense operator
    hv = op(psi).data
    assert np.linalg.norm(hv - H @ pd) <= 1e-12 * np.linalg.norm(H @ pd)


def test_lanczos_converges_to_exact_ground_state():
    from sparsebackends_b200 import krylov
    sb, lay, op, psi, pd, H = _heff_problem(23)
    ev = np.linalg.eigh(H)[0]
    vals, vecs, info = krylov.eigsolve(op, psi, 1, "SR", krylovdim=20, maxiter=300, tol=1e-10)
    assert info.converged >= 1
    assert abs(vals[0] - ev[0]) <= 1e-9 * abs(ev[0])
    v = vecs[0]
    res = op(v) - vals[0] * v
    assert sb.norm(res) <= 1e-8 * abs(vals[0]) * sb.norm(v)
    # the restarted device solve follows the oracle's restarted solve
    rv, *_ = ko.lanczos_eigsolve(lambda x: H @ x, pd, 1, "SR", krylovdim=20, maxiter=300, tol=1e-10)
    assert abs(vals[0] - rv[0]) <= 1e-10 * abs(rv[0])
