"""The PXP chain's step tables (``sparsebackends_b200.pxp``) on the oracle,
against a dense einsum restatement of the same Hamiltonian, at small sizes.

The device path runs these tables unchanged (``tests/test_gpu_pxp_heff.py``);
here they are checked for the label flow (every contraction is one the
reference's kernels accept: no tail permutes, fused pairs adjacent) and for the
physics (H_eff symmetric, the MPO's boundary channels)."""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from sparsebackends_b200 import pxp
from tests import pxp_ref as pr

N, CHI, SEED = 12, 16, 5


@pytest.fixture(scope="module")
def prob():
    return pr.OracleProblem(N, CHI, SEED)


def test_mpo_is_pxp():
    """Contracting the MPO along a 4-site chain gives sum_i P X P on the two
    interior sites."""
    Wd = pxp.mpo_dense()
    n = 4
    H = np.zeros((1, 1, pxp.W))
    H[0, 0, pxp.LEFT_CHANNEL - 1] = 1.0
    for _ in range(n):
        H = np.einsum("abw,xywv->axbyv", H, Wd).reshape(H.shape[0] * 2, H.shape[1] * 2, pxp.W)
    H = H[:, :, pxp.RIGHT_CHANNEL - 1]
    P, X, I = pxp.OPS["P"], pxp.OPS["X"], np.eye(2)

    def kron(*ops):
        out = np.ones((1, 1))
        for o in ops:
            out = np.kron(out, o)
        return out
    # the sum is symmetric under reversing the chain, so the site order of
    # the Kronecker products does not matter
    want = np.zeros((2 ** n, 2 ** n))
    for i in range(1, n - 1):
        ops = [I] * n
        ops[i - 1], ops[i], ops[i + 1] = P, X, P
        want += kron(*reversed(ops))
    assert np.array_equal(H, want)


def test_mpo_coo_has_eight_entries():
    keys, vals = pxp.mpo_entries()
    assert len(keys) == 8 and set(vals) == {1.0}
    assert len({(k[2], k[3]) for k in keys}) == 5


def test_sites_are_canonical(prob):
    for k in range(1, prob.c):
        A = prob.sites[k - 1]
        m = A.reshape(-1, A.shape[2], order="F")
        assert np.allclose(m.T @ m, np.eye(A.shape[2]), atol=1e-12)
    for k in range(N, prob.c + 1, -1):
        B = prob.sites[k - 1]
        m = B.reshape(B.shape[0], -1, order="F")
        assert np.allclose(m @ m.T, np.eye(B.shape[0]), atol=1e-12)


def test_environments_match_dense(prob):
    Ld = pr.dense_env_L(prob.sites, prob.c)
    Rd = pr.dense_env_R(prob.sites, N, prob.c)
    assert np.allclose(pr.env_to_dense(prob.L, right=False), Ld, rtol=0, atol=1e-12)
    assert np.allclose(pr.env_to_dense(prob.R, right=True), Rd, rtol=0, atol=1e-12)


def test_heff_matches_dense(prob):
    out = prob.apply(prob.psi)
    assert out.dims == prob.psi.dims
    got = pr.psi_to_dense(out)
    Ld = pr.dense_env_L(prob.sites, prob.c)
    Rd = pr.dense_env_R(prob.sites, N, prob.c)
    want = pr.dense_heff(Ld, Rd, prob.psi_host)
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_heff_is_symmetric(prob):
    rng = np.random.Generator(np.random.PCG64(9))
    phi_h = rng.standard_normal(prob.psi_host.shape)
    phi = pr.o_bs(*pxp.psi_blocks(phi_h))
    a = so.bs_dot(phi, prob.apply(prob.psi))
    b = so.bs_dot(prob.apply(phi), prob.psi)
    assert abs(a - b) <= 1e-12 * max(abs(a), 1.0)


def test_both_join_orders_agree(prob):
    """Every contract_shared! of the tables joins on one axis of extent > 1,
    so the reference's merge order gives the same result."""
    base = prob.apply(prob.psi)
    with so.join_order("reference"):
        ref = prob.apply(prob.psi)
    assert base.keys == ref.keys
    for i, j in zip(base.ids, ref.ids):
        assert np.array_equal(base.block(i), ref.block(j))


def test_aliased_heff_matches_dense(prob):
    """The aliased form (W as templates I, P, X; dense psi and environments)
    gives the same H_eff . psi."""
    X4 = prob.apply_aliased(prob.psi_host)
    assert X4.keys == [()]
    got = X4.logical_blocks()[()].reshape(prob.psi_host.shape, order="F")
    want = pr.dense_heff(pr.dense_env_L(prob.sites, prob.c), pr.dense_env_R(prob.sites, N, prob.c), prob.psi_host)
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    dims, tm, keys, aids, sc = pxp.mpo_aliased()
    assert len(keys) == 5 and len(tm) == 3 * pxp.D * pxp.D
