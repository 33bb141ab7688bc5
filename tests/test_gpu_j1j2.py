"""Two-site DMRG (``dmrg.DMRG``) on the J1-J2 cylinder MPO
(``j1j2.J1J2Cylinder``): the ground-state energy of small cylinders against
exact diagonalisation of the 2Sz = 0 sector, in FP64 and in the 3xTF32 form."""
import pytest

from sparsebackends_b200 import j1j2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as sbmod
    return sbmod


@pytest.mark.parametrize("lx,ly", [(3, 4), (2, 6)])
@pytest.mark.parametrize("precision", ["f64", "tf32x3"])
def test_j1j2_ground_energy(sb, lx, ly, precision):
    from sparsebackends_b200 import dmrg
    m = j1j2.J1J2Cylinder(lx, ly, 1.0, 0.5)
    exact = j1j2.exact_ground_energy(m.n, m.J)
    d = dmrg.DMRG(m.n, ctx=sb.Context(0), precision=precision, mpo=m)
    e, _ = d.run([16, 32, 64] + [64] * 7, cutoff=1e-14, krylovdim=8, maxiter=3)
    assert abs(e - exact) <= 1e-9 * abs(exact), (e, exact)


def test_j1j2_gram_split(sb):
    """The sweep with the density-matrix split (method "gram") reaches the
    same exact energy."""
    from sparsebackends_b200 import dmrg
    m = j1j2.J1J2Cylinder(3, 4, 1.0, 0.5)
    exact = j1j2.exact_ground_energy(m.n, m.J)
    d = dmrg.DMRG(m.n, ctx=sb.Context(0), device_split=True, mpo=m, split_method="gram")
    e, _ = d.run([16, 32, 64] + [64] * 7, cutoff=1e-14, krylovdim=8, maxiter=3)
    assert abs(e - exact) <= 1e-9 * abs(exact), (e, exact)
