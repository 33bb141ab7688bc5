"""GPU parity of the block factorisations against the oracle (ops_factorize.jl).

* blocksparse_left_qr: Householder QR on the device with LAPACK's reflector
  sign convention, so Q blocks and R match numpy's LAPACK QR entry by entry
  (1e-12); l/r value lists exact; rank-deficient inputs checked by
  reconstruction and orthogonality.
* blocksparse_svd: singular values (1e-12 relative), bond structure (keys of
  U and SV) and truncation error exact against the oracle's truncation; U and
  SV blocks equal up to the sign of each singular pair (gauge), 1e-10;
  U·SV reproduces the truncated input.
"""
import numpy as np
import pytest

from oracle import factorize_oracle as fo
from oracle import sparse_oracle as so

pytestmark = pytest.mark.gpu


def _sb():
    import sparsebackends_b200 as sb
    return sb


def _dev(sb, X, ctx):
    return sb.NewBlockSparseSorted(X.dims, X.n2, X.keys, X.ids, X.data, ctx=ctx)


def _host(T, n2):
    """Device block-sparse tensor -> oracle BS (ids 1..n in key order)."""
    keys = T.keys
    return so.BS(T.dims, n2, keys, list(range(1, len(keys) + 1)), T.data)


def _bs(seed, dims, n2, p):
    rng = np.random.Generator(np.random.PCG64(seed))
    P = len(dims) - n2
    D = rng.standard_normal(dims) * (rng.random(dims[:P] + (1,) * n2) < p)
    D[(0,) * P] += 1.0
    return D, so.blocksparse_from_dense(D, n2)


@pytest.mark.parametrize("seed,dims,p", [(0, (6, 5, 3), 0.6), (1, (9, 4, 2), 0.7), (2, (3, 12, 4), 0.8),
                                         (3, (40, 30, 2), 0.3)])
def test_left_qr_matches_lapack(seed, dims, p):
    sb = _sb()
    ctx = sb.Context(0)
    D, A = _bs(seed, dims, 1, p)
    Qr, Rr, lr, rr = fo.blocksparse_left_qr(A)
    Q, R, lv, rv = sb.blocksparse_left_qr(_dev(sb, A, ctx))
    assert (lv, rv) == (lr, rr)
    assert Q.dims == Qr.dims and Q.keys == Qr.keys
    qb, qrb = Q.blocks_by_key(), Qr.blocks_by_key()
    for k in qrb:
        assert np.allclose(qb[k], qrb[k], atol=1e-12, rtol=0), k
    assert np.allclose(R.to_numpy(), Rr, atol=1e-12 * max(1.0, np.abs(Rr).max()), rtol=0)


def test_left_qr_rank_deficient():
    sb = _sb()
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(5))
    D = np.zeros((4, 6, 2))
    base = rng.standard_normal((4, 2))
    for r in range(6):
        D[:, r, :] = base * (r % 2 + 1)  # rank 1 across r
    A = so.blocksparse_from_dense(D, 1)
    Q, R, lv, rv = sb.blocksparse_left_qr(_dev(sb, A, ctx))
    Qd = so.bs_to_dense(_host(Q, 2))
    Qm = np.concatenate([Qd[l - 1] for l in lv], axis=0)
    M = np.stack([np.concatenate([D[l - 1, r - 1, :] for l in lv]) for r in rv], axis=1)
    assert np.allclose(Qm @ R.to_numpy(), M, atol=1e-12)
    assert np.allclose(Qm.T @ Qm, np.eye(Qm.shape[1]), atol=1e-12)


def _canon(U, SV, nb):
    """Fix the sign of each singular pair: the largest-|.| entry of U's column
    b is made positive; the same sign flips SV's row b."""
    ub, vb = U.blocks_by_key(), SV.blocks_by_key()
    sign = {}
    for b in range(1, nb + 1):
        entries = np.concatenate([v for k, v in ub.items() if k[1] == b])
        sign[b] = 1.0 if entries[np.argmax(np.abs(entries))] >= 0 else -1.0
    return ({k: v * sign[k[1]] for k, v in ub.items()}, {k: v * sign[k[0]] for k, v in vb.items()})


@pytest.mark.parametrize("ortho", ["left", "right"])
@pytest.mark.parametrize("seed,dims,p,kw", [
    (10, (5, 6, 2, 3), 0.5, {}),
    (11, (8, 7, 3, 2), 0.4, {"cutoff": 1e-2}),
    (12, (6, 9, 2, 2), 0.6, {"maxdim": 5}),
    (13, (12, 3, 4, 1), 0.7, {"maxdim": 7, "mindim": 6, "cutoff": 0.3}),
    (14, (30, 40, 2, 2), 0.3, {"cutoff": 1e-10}),
])
def test_svd_matches_oracle(ortho, seed, dims, p, kw):
    sb = _sb()
    ctx = sb.Context(0)
    D, A = _bs(seed, dims, 2, p)
    Ur, SVr, kr, (er, ter) = fo.blocksparse_svd(A, ortho=ortho, **kw)
    U, SV, kept, spec = sb.blocksparse_svd(_dev(sb, A, ctx), ortho=ortho, **kw)
    assert len(kept) == len(kr)
    assert np.allclose(kept, kr, rtol=1e-12, atol=1e-14 * kr.max())
    assert abs(spec["truncerr"] - ter) <= 1e-12 * max(ter, 1e-300) + 1e-28
    assert U.dims == Ur.dims and SV.dims == SVr.dims
    assert U.keys == Ur.keys and SV.keys == SVr.keys
    ug, vg = _canon(U, SV, len(kept))
    ur, vr = _canon(Ur, SVr, len(kr))
    for k in ur:
        assert np.allclose(ug[k], ur[k], atol=1e-10), k
    for k in vr:
        assert np.allclose(vg[k], vr[k], atol=1e-10 * max(1.0, kr.max())), k
    # U·SV = the truncated input (equal to A when nothing is dropped)
    Ud = so.bs_to_dense(_host(U, 1))
    Vd = so.bs_to_dense(_host(SV, 1))
    rec = np.einsum("lbs,brt->lrst", Ud, Vd)
    Urd = so.bs_to_dense(Ur)
    Vrd = so.bs_to_dense(SVr)
    assert np.allclose(rec, np.einsum("lbs,brt->lrst", Urd, Vrd), atol=1e-10)


def test_factorize_errors():
    sb = _sb()
    ctx = sb.Context(0)
    _, A = _bs(20, (4, 4, 2, 2), 2, 0.5)
    with pytest.raises(sb.SparseBackendsError) as e:
        sb.blocksparse_left_qr(_dev(sb, A, ctx))
    assert e.value.code == 4  # SB_ERR_UNSUPPORTED_LAYOUT: not (l, r | s)
    _, B = _bs(21, (4, 4, 3), 1, 0.5)
    with pytest.raises(sb.SparseBackendsError) as e:
        sb.blocksparse_svd(_dev(sb, B, ctx))
    assert e.value.code == 4
