"""CPU checks of the factorisation oracle (ops_factorize.jl restated).

* blocksparse_left_qr: Q R reproduces the assembled matrix, Q has orthonormal
  columns, one Q block per distinct l value;
* blocksparse_svd: U·SV reproduces A without truncation; the global
  truncation rule on hand-placed singular values (known answers: keep counts,
  bond order, truncerr) for cutoff, maxdim and mindim.
"""
import numpy as np
import pytest

from oracle import factorize_oracle as fo
from oracle import sparse_oracle as so


def _bs3(seed, dims=(6, 5, 3), p=0.5):
    rng = np.random.Generator(np.random.PCG64(seed))
    D = rng.standard_normal(dims) * (rng.random(dims[:2] + (1,)) < p)
    D[0, 0, :] += 1.0  # at least one block
    return D, so.blocksparse_from_dense(D, 1)


def _dense(T):
    return so.bs_to_dense(T)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_left_qr_reconstructs(seed):
    D, A = _bs3(seed)
    Q, R, lv, rv = fo.blocksparse_left_qr(A)
    ds = D.shape[2]
    M = np.zeros((len(lv) * ds, len(rv)))
    for a, l in enumerate(lv):
        for b, r in enumerate(rv):
            M[a * ds:(a + 1) * ds, b] = D[l - 1, r - 1, :]
    Qd = _dense(Q)  # (nl_total, ds, k)
    Qm = np.concatenate([Qd[l - 1] for l in lv], axis=0)
    assert np.allclose(Qm @ R, M, atol=1e-12)
    assert np.allclose(Qm.T @ Qm, np.eye(Qm.shape[1]), atol=1e-12)
    assert sorted(k[0] for k in Q.keys) == lv


def _bs4(seed, dims=(5, 6, 2, 3), p=0.5):
    rng = np.random.Generator(np.random.PCG64(seed))
    D = rng.standard_normal(dims) * (rng.random(dims[:2] + (1, 1)) < p)
    D[0, 0] += 1.0
    return D, so.blocksparse_from_dense(D, 2)


@pytest.mark.parametrize("ortho", ["left", "right"])
@pytest.mark.parametrize("seed", [3, 4])
def test_svd_reconstructs_without_truncation(ortho, seed):
    D, A = _bs4(seed)
    U, SV, kept, (eigs, te) = fo.blocksparse_svd(A, ortho=ortho)
    Ud, Vd = _dense(U), _dense(SV)
    rec = np.einsum("lbs,brt->lrst", Ud, Vd)
    assert np.allclose(rec, D, atol=1e-12)
    assert te < 1e-24
    assert np.allclose(eigs, kept ** 2)


def _diag_case():
    """Groups L=1: svs (3, 1e-3) from (R=1), L=2: (2, 5e-11) from (R=2),
    L=3: (0.5,) (single column), as diagonal 2 x 2 blocks."""
    D = np.zeros((3, 3, 2, 2))
    D[0, 0] = np.diag([3.0, 1e-3])
    D[1, 1] = np.diag([2.0, 5e-11])
    D[2, 2] = np.diag([0.5, 0.0])
    return so.blocksparse_from_dense(D, 2)


def test_truncation_known_answers():
    A = _diag_case()
    # cutoff 1e-10 drops 5e-11 and the zero: kept [3, 1e-3 | 2 | 0.5] in group order
    U, SV, kept, (_, te) = fo.blocksparse_svd(A, cutoff=1e-10)
    assert np.allclose(kept, [3.0, 1e-3, 2.0, 0.5])
    assert abs(te - (5e-11) ** 2) < 1e-30
    assert [k for k in U.keys] == [(1, 1), (1, 2), (2, 3), (3, 4)]
    # maxdim 2: the two largest (3 and 2), one per group 1 and 2
    U, SV, kept, (_, te) = fo.blocksparse_svd(A, maxdim=2)
    assert np.allclose(kept, [3.0, 2.0])
    assert abs(te - (1e-6 + 0.25 + (5e-11) ** 2)) < 1e-15
    # cutoff 0.5 keeps 3 and 2 (0.5*3 = 1.5 > 0.5, 1e-3); mindim 3 forces the third
    _, _, kept, _ = fo.blocksparse_svd(A, cutoff=0.5)
    assert np.allclose(kept, [3.0, 2.0])
    _, _, kept, _ = fo.blocksparse_svd(A, cutoff=0.5, mindim=3)
    assert np.allclose(kept, [3.0, 2.0, 0.5])
