"""Mixed-precision DMRG: the Lanczos H_eff applies on the tcgen05 tensor cores
(3xTF32 block GEMMs, FP32 intermediates), everything else FP64, and each bond's
energy the FP64 Rayleigh quotient of its Ritz vector (the FP64 residual
correction of ``krylov.eigsolve(..., correction=)``).

Against the FP64 DMRG on the same chain and the same sweep schedule (the
FP64 run is the oracle of the mixed form): the final energies agree to
ENERGY_RTOL relative, and the FP64 energy equals the exact ground-state
energy of the 2Sz = 0 sector to 1e-9.
"""
import pytest

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-10


@pytest.mark.parametrize("n,delta", [(8, 1.0), (10, 1.0), (10, 0.5)])
def test_mixed_dmrg_energy_matches_fp64(n, delta):
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg
    sched = [4, 16, 32, 32, 32, 32]
    ref = dmrg.DMRG(n, delta, sb.Context(0))
    e64, es64 = ref.run(sched, cutoff=1e-14, krylovdim=8, maxiter=3)
    mix = dmrg.DMRG(n, delta, sb.Context(0), precision="tf32x3")
    emx, esmx = mix.run(sched, cutoff=1e-14, krylovdim=8, maxiter=3)
    exact = dmrg.exact_ground_energy(n, delta)
    assert abs(e64 - exact) <= 1e-9 * abs(exact), (e64, exact)
    assert abs(emx - e64) <= ENERGY_RTOL * abs(e64), (emx, e64, esmx, es64)


def test_mixed_eigsolve_correction_on_heisenberg_heff():
    """One H_eff of the N = 8 Heisenberg chain (environments from a converged
    FP64 DMRG): the 3xTF32 Lanczos with the FP64 correction finds the FP64
    Lanczos energy to ENERGY_RTOL, and its FP64 residual is small."""
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg, krylov, qn
    ctx = sb.Context(0)
    d = dmrg.DMRG(8, 1.0, ctx)
    d.run([16, 16, 16], cutoff=1e-14, krylovdim=8, maxiter=3)
    i = 4
    lay, x = d._two_site(i)
    args = (lay, d.Lenv[i - 1], d.Ws[i - 1], d.Ws[i], d.Renv[i + 1], ctx)
    op64 = qn.HeffOperator(*args)
    opmx = qn.HeffOperator(*args, precision="tf32x3")
    v64, _, _ = krylov.eigsolve(op64, x, 1, "SR", krylovdim=12, maxiter=4, tol=1e-14)
    vmx, vecs, info = krylov.eigsolve(opmx, x, 1, "SR", krylovdim=12, maxiter=4, tol=1e-14, correction=op64,
                                      optol=opmx.accuracy)
    assert abs(vmx[0] - v64[0]) <= ENERGY_RTOL * abs(v64[0]), (vmx, v64)
    assert info.residuals and info.residuals[0] < 1e-4, info.residuals
    assert ctx.precision == "f64"  # the operator restores the context precision
