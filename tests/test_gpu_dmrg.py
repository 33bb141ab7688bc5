"""Two-site DMRG on the device (``sparsebackends_b200.dmrg``): the XXZ chain
from the Néel state, sweeps of ψ = A·A, device Lanczos on H_eff, U(1) split and
environment updates, against exact diagonalisation of the 2Sz = 0 sector.

* Heisenberg (Δ = 1), N = 8 and 10: the energy after the sweeps equals the
  exact ground-state energy (1e-9 relative) with the bond dimension allowed to
  reach the exact one;
* XXZ Δ = 0.5, N = 8: the same;
* with the reference's Lanczos setting (krylovdim 3, maxiter 1 per bond) the
  energy still converges (1e-6 relative after eight sweeps) and never rises by
  more than rounding between sweeps.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,delta", [(8, 1.0), (10, 1.0), (8, 0.5)])
def test_dmrg_matches_exact_diagonalisation(n, delta):
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg
    d = dmrg.DMRG(n, delta, sb.Context(0))
    e, es = d.run([4, 16, 32, 32, 32, 32], cutoff=1e-14, krylovdim=8, maxiter=3)
    exact = dmrg.exact_ground_energy(n, delta)
    assert abs(e - exact) <= 1e-9 * abs(exact), (e, exact, es)


def test_dmrg_reference_lanczos_setting_converges():
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg
    d = dmrg.DMRG(8, 1.0, sb.Context(0))
    e, es = d.run([8, 16] + [16] * 6, cutoff=1e-12, krylovdim=3, maxiter=1)
    exact = dmrg.exact_ground_energy(8, 1.0)
    assert abs(e - exact) <= 1e-6 * abs(exact), (e, exact, es)
    assert all(b <= a + 1e-10 for a, b in zip(es, es[1:])), es


def test_device_split_matches_host_split():
    """qn.split_two_site_device (SVD per centre charge on the GPU) against the
    host split on the same two-site tensor: the same bond sectors, singular
    values to 1e-12, and A*B reproducing the truncated psi of the host split."""
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    ctx = sb.Context(0)
    left = qn.U1Link([-3, -1, 1, 3], [3, 9, 9, 3])
    right = qn.U1Link([-3, -1, 1, 3], [5, 11, 11, 5])
    lay = qn.HeffLayout(left, right, qn.mpo_link({-2: 1, 0: 3, 2: 1}))
    keys, data, exts = qn.random_block_tensor(lay, "psi", np.random.Generator(np.random.PCG64(17)), 1.0,
                                              ragged=True)
    psi = sb.NewBlockSparseSorted(lay.dims["psi"], lay.n2["psi"], keys, None, data, ctx=ctx, block_dims=exts)
    for absorb in ("right", "left"):
        (ak, ad, ae), (bk, bd, be), link_h, sv_h, err_h = qn.split_two_site(lay, keys, data, exts, maxdim=20,
                                                                           cutoff=1e-3, absorb=absorb)
        A, B, link_d, sv_d, err_d = qn.split_two_site_device(lay, psi, maxdim=20, cutoff=1e-3, absorb=absorb)
        assert link_d.charges == link_h.charges and link_d.dims == link_h.dims
        assert np.allclose(sv_d, sv_h, rtol=1e-12, atol=0) and abs(err_d - err_h) <= 1e-12
        assert A.keys == ak and B.keys == bk
        Ah = sb.NewBlockSparseSorted(A.dims, 2, ak, None, ad, ctx=ctx, block_dims=ae)
        Bh = sb.NewBlockSparseSorted(B.dims, 2, bk, None, bd, ctx=ctx, block_dims=be)
        lab = (["ql", "s1", "s2", "qr", "ml", "mr"], ["ql", "s1", "qc", "ml", "mc"], ["qc", "s2", "qr", "mc", "mr"])
        pd = qn.contract_new(lab[0], 2, A, lab[1], B, lab[2])
        ph = qn.contract_new(lab[0], 2, Ah, lab[1], Bh, lab[2])
        assert pd.keys == ph.keys
        gd, gh = pd.blocks_by_key(), ph.blocks_by_key()
        nrm = np.linalg.norm(np.array(ph.data))
        assert max(np.abs(np.asarray(gd[k]) - np.asarray(v)).max() for k, v in gh.items()) <= 1e-12 * nrm


def test_dmrg_device_split_energy():
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg
    sched = [4, 16, 32, 32, 32, 32]
    e_d, _ = dmrg.DMRG(10, 1.0, sb.Context(0), device_split=True).run(sched, cutoff=1e-14, krylovdim=8, maxiter=3)
    e_h, _ = dmrg.DMRG(10, 1.0, sb.Context(0), device_split=False).run(sched, cutoff=1e-14, krylovdim=8, maxiter=3)
    assert abs(e_d - e_h) <= 1e-12 * abs(e_h), (e_d, e_h)
    exact = dmrg.exact_ground_energy(10, 1.0)
    assert abs(e_d - exact) <= 1e-9 * abs(exact)


def test_device_split_gram_matches_svd():
    """The density-matrix split (method="gram": eigh of M M^T or M^T M) against
    the SVD split on the same two-site tensor: the same bond sectors, singular
    values to 1e-10 of the largest, the same discarded weight, the isometry
    orthonormal to 1e-12 and A*B equal to the SVD truncation's to 1e-10."""
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    ctx = sb.Context(0)
    left = qn.U1Link([-3, -1, 1, 3], [3, 9, 9, 3])
    right = qn.U1Link([-3, -1, 1, 3], [5, 11, 11, 5])
    lay = qn.HeffLayout(left, right, qn.mpo_link({-2: 1, 0: 3, 2: 1}))
    keys, data, exts = qn.random_block_tensor(lay, "psi", np.random.Generator(np.random.PCG64(23)), 1.0,
                                              ragged=True)
    psi = sb.NewBlockSparseSorted(lay.dims["psi"], lay.n2["psi"], keys, None, data, ctx=ctx, block_dims=exts)
    lab = (["ql", "s1", "s2", "qr", "ml", "mr"], ["ql", "s1", "qc", "ml", "mc"], ["qc", "s2", "qr", "mc", "mr"])
    for absorb in ("right", "left"):
        A1, B1, l1, sv1, e1 = qn.split_two_site_device(lay, psi, maxdim=20, cutoff=1e-3, absorb=absorb)
        A2, B2, l2, sv2, e2 = qn.split_two_site_device(lay, psi, maxdim=20, cutoff=1e-3, absorb=absorb,
                                                       method="gram")
        assert l1.charges == l2.charges and l1.dims == l2.dims
        assert np.allclose(sv2, sv1, rtol=0, atol=1e-10 * sv1[0]) and abs(e1 - e2) <= 1e-12
        p1 = qn.contract_new(lab[0], 2, A1, lab[1], B1, lab[2]).blocks_by_key()
        p2 = qn.contract_new(lab[0], 2, A2, lab[1], B2, lab[2]).blocks_by_key()
        assert set(p1) == set(p2)
        nrm = np.sqrt(sum(float(np.sum(np.asarray(v) ** 2)) for v in p1.values()))
        assert max(np.abs(np.asarray(p2[k]) - np.asarray(v)).max() for k, v in p1.items()) <= 1e-10 * nrm
        # the isometry: A's rows (absorb right) or B's columns (absorb left) orthonormal per bond sector
        iso = A2 if absorb == "right" else B2
        blocks = iso.blocks_by_key()
        dims = dict(zip(iso.keys, iso.block_dims))
        for qc in range(1, l2.S + 1):
            if absorb == "right":
                parts = [np.asarray(blocks[k]).reshape(dims[k], order="F") for k in iso.keys if k[2] == qc]
                Q = np.vstack(parts)
            else:
                parts = [np.asarray(blocks[k]).reshape(dims[k], order="F") for k in iso.keys if k[0] == qc]
                Q = np.hstack(parts).T
            assert np.allclose(Q.T @ Q, np.eye(Q.shape[1]), atol=1e-12)
