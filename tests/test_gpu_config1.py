"""The two-site H_eff of a canonical Heisenberg MPS, the reference's CPU
matvec case: N = 16, open chain, U(1) on 2Sz, the centre bond between sites 8
and 9, chi = 64 with the centre link's sectors 2Sz = -4..4 at
{4, 12, 32, 12, 4} and the other links capped at their Hilbert-space bound.

``dmrg.canonical_center_problem`` fills every allowed block with seeded
N(0, 1) entries, left-canonicalises sites 1..7 and right-canonicalises sites
10..16 by the library's ``blocksparse_left_qr`` (ops_factorize.jl:8-43) per
charge sector, builds L and R from the boundaries by ``make_L`` / ``make_R``
(three ``contract!`` calls each) and draws psi Gaussian on the flux-0 blocks
of sites 8 and 9, normalised.

Checked:

* canonical form: the identity channel of L (of R) is the identity matrix on
  every sector of the link, to 1e-12;
* the GPU chain's output keys equal the oracle's four-step chain on the
  zero-padded (reference-layout) operands, every block to 1e-12 relative
  Frobenius error on the FP64 path and to 2e-5 with 3xTF32 tensor-core GEMMs
  and FP32 intermediates;
* H_eff is symmetric: <phi, H psi> = <H phi, psi> to 1e-12 (relative to
  |H psi| |phi|).
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12
TOL_X3 = 2e-5


@pytest.fixture(scope="module")
def problem():
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg, qn
    ctx = sb.Context(0)
    lay, psi, L, W, R = dmrg.canonical_center_problem(ctx)
    return sb, qn, dmrg, ctx, lay, psi, L, W, R


def _padded(sb, t):
    u = sb.to_uniform(t)
    return so.BS(u.dims, u.n2, u.keys, list(range(1, len(u.keys) + 1)), np.array(u.data, copy=True))


@pytest.fixture(scope="module")
def oracle_out(problem):
    sb, qn, dmrg, ctx, lay, psi, L, W, R = problem
    t = {"psi": _padded(sb, psi), "L": _padded(sb, L), "W1": _padded(sb, W), "W2": _padded(sb, W),
         "R": _padded(sb, R)}
    lab = lay.labels
    for c, a, b in qn.HeffChain.STEPS:
        t[c] = so.contract(so.BS.empty(lay.dims[c], lay.n2[c]), lab[c], t[a], lab[a], t[b], lab[b])
    return t["T4"]


def test_links(problem):
    sb, qn, dmrg, ctx, lay, psi, L, W, R = problem
    centre = dmrg.profile_link(16, 8)
    assert centre.charges == [-4, -2, 0, 2, 4] and centre.dims == [4, 12, 32, 12, 4]
    assert lay.left.charges == [-3, -1, 1, 3] and lay.left.dims == [8, 22, 22, 8]
    assert lay.right.charges == lay.left.charges and lay.right.dims == lay.left.dims
    for b in range(17):
        assert max(dmrg.profile_link(16, b).dims) <= 32 and sum(dmrg.profile_link(16, b).dims) <= 64


def _identity_channel(env, link, channel, dmrg):
    q0 = dmrg.MPO_LINK.index(0) + 1
    m = dmrg.CHANNEL[channel][1] - 1
    blocks = env.blocks_by_key()
    for a, d in enumerate(link.dims, start=1):
        blk = np.asarray(blocks[(a, q0, a)]).reshape((d, dmrg.MPO_LINK.dims[q0 - 1], d), order="F")
        assert np.abs(blk[:, m, :] - np.eye(d)).max() <= 1e-12, (a, channel)


def test_canonical_environments(problem):
    sb, qn, dmrg, ctx, lay, psi, L, W, R = problem
    _identity_channel(L, lay.left, 1, dmrg)   # "identity before" channel of the left environment
    _identity_channel(R, lay.right, 5, dmrg)  # "identity after" channel of the right environment


def _check(sb, out, ref, tol):
    got = sb.to_uniform(out)
    assert got.keys == ref.keys and len(ref.keys) > 0
    gb, rb = got.blocks_by_key(), ref.blocks_by_key()
    worst = 0.0
    for k, v in rb.items():
        e = float(np.linalg.norm(np.asarray(gb[k]) - v) / max(np.linalg.norm(v), 1e-300))
        worst = max(worst, e)
        assert e <= tol, (k, e)
    return worst


def test_chain_matches_oracle(problem, oracle_out):
    sb, qn, dmrg, ctx, lay, psi, L, W, R = problem
    out = qn.HeffChain(lay, ctx).apply(psi, L, W, W, R)
    _check(sb, out, oracle_out, TOL_F64)


@pytest.mark.parametrize("w12", [False, True])
def test_tensor_core_chain_matches_oracle(problem, oracle_out, w12):
    sb, qn, dmrg, ctx, lay, psi, L, W, R = problem
    cm = sb.Context(0)
    cm.set_precision("tf32x3")
    # the operands built on the FP64 context, copied over
    psi2, L2, W2, R2 = (sb.NewBlockSparseSorted(t.dims, t.n2, t.keys, None, np.array(t.data), ctx=cm,
                                                block_dims=t.block_dims) for t in (psi, L, W, R))
    out = qn.HeffChain(lay, cm, w12=w12, f32_intermediates=True).apply(psi2, L2, W2, W2, R2)
    cm.synchronize()
    worst = _check(sb, out, oracle_out, TOL_X3)
    print(f"config 1 tf32x3 w12={w12}: worst block rel err vs oracle {worst:.2e}")


def test_symmetric(problem):
    sb, qn, dmrg, ctx, lay, psi, L, W, R = problem
    op = qn.HeffOperator(lay, L, W, W, R, ctx)
    keys, data, exts = qn.random_block_tensor(lay, "psi", np.random.Generator(np.random.PCG64(9)), 1.0,
                                              ragged=True)
    phi = sb.NewBlockSparseSorted(lay.dims["psi"], lay.n2["psi"], keys, None, data, ctx=ctx, block_dims=exts)
    assert phi.keys == psi.keys
    hpsi, hphi = op(psi), op(phi)

    def dot(x, y):
        yb = y.blocks_by_key()
        return sum(float(np.dot(np.ravel(v), np.ravel(yb[k]))) for k, v in x.blocks_by_key().items() if k in yb)

    a, b = dot(phi, hpsi), dot(hphi, psi)
    scale = np.linalg.norm(np.array(hpsi.data)) * np.linalg.norm(np.array(phi.data))
    assert abs(a - b) <= 1e-12 * scale
