"""The J1-J2 cylinder MPO (``sparsebackends_b200.j1j2``): contracted along the
chain it equals the Hamiltonian built from the couplings, and the couplings
are those of the lattice."""
import numpy as np
import pytest

from sparsebackends_b200 import j1j2, qn


def test_couplings_of_a_6x6_cylinder():
    J = j1j2.cylinder_couplings(6, 6, 1.0, 0.5)
    n1 = sum(1 for v in J.values() if v == 1.0)
    n2 = sum(1 for v in J.values() if v == 0.5)
    assert n1 == 6 * 6 + 5 * 6  # vertical rings + horizontal rungs
    assert n2 == 2 * 5 * 6      # two diagonals per plaquette column
    assert all(i < j for i, j in J)
    # snake order: site (1, 0) follows (0, 5)
    assert j1j2.snake_index(0, 5, 6) == 5 and j1j2.snake_index(1, 5, 6) == 6


def test_link_size_of_a_6x6_cylinder():
    m = j1j2.J1J2Cylinder(6, 6)
    w = m.link
    assert w.charges == [-2, 0, 2]
    assert w.dims[0] == w.dims[2] and w.dims[1] == w.dims[0] + 2
    assert 20 <= w.total <= 60


def _contract(m):
    l, r = m.boundary_vectors()
    acc = [np.ones((1, 1)) * x for x in l]  # per left channel, the operator so far
    for k in range(m.n):
        Wk = m.dense_mpo(k)
        nxt = []
        for wr in range(Wk.shape[1]):
            tot = None
            for wl in range(Wk.shape[0]):
                op = Wk[wl, wr]
                if not op.any() or not acc[wl].any():
                    continue
                t = np.kron(acc[wl], op)
                tot = t if tot is None else tot + t
            nxt.append(tot if tot is not None else np.zeros((2 ** (k + 1), 2 ** (k + 1))))
        acc = nxt
    return sum(r[w] * acc[w] for w in range(len(acc)) if r[w] != 0.0)


@pytest.mark.parametrize("lx,ly", [(2, 3), (3, 2), (2, 4)])
def test_mpo_equals_hamiltonian(lx, ly):
    m = j1j2.J1J2Cylinder(lx, ly, 1.0, 0.5)
    H = _contract(m)
    want = j1j2.dense_hamiltonian(m.n, m.J)
    assert np.allclose(H, want, atol=1e-13, rtol=0)


def test_blocks_conserve_charge():
    m = j1j2.J1J2Cylinder(3, 4)
    w = m.link
    for k in range(m.n):
        for (ql, sp, s, qr) in m.site_blocks(k):
            assert w.charges[qr - 1] == w.charges[ql - 1] + qn.PHYS[sp - 1] - qn.PHYS[s - 1]


def test_narrow_cylinder_counts_each_pair_once():
    """On a width-2 cylinder the periodic wrap meets the direct bond: one J1
    per rung, one J1 per leg bond and one J2 per diagonal."""
    J = j1j2.cylinder_couplings(3, 2, 1.0, 0.5)
    assert sum(1 for v in J.values() if v == 1.0) == 3 + 2 * 2   # rungs + legs
    assert sum(1 for v in J.values() if v == 0.5) == 2 * 2       # two diagonals per plaquette
    assert set(J.values()) == {1.0, 0.5}
