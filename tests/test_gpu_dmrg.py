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
