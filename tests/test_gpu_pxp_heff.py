"""The PXP chain on the device (``sparsebackends_b200.pxp``) against the oracle
running the same step tables (``tests/pxp_ref.py``): environments built from
the boundaries, the two-site H_eff matvec with the MPO in COO, in the plain
FP64 form and the 3xTF32 form, and the MPO x MPS apply on every site tensor.

Sizes: N = 64, chi = 256 (the PXP benchmark shapes) and a small N = 12,
chi = 16 chain.  The COO steps (scaled block adds by the MPO's 0/1 entries)
round like the oracle; the dense contractions sum in a different order than
numpy, so FP64 results agree to 1e-13 relative, not bit for bit.  The 3xTF32
form is held to 1e-5 relative (max abs error over max abs value), the bound the
tensor-core contractions are specified to."""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from sparsebackends_b200 import pxp
from tests import pxp_ref as pr

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-13
TF32X3_RTOL = 1e-5


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as sbmod
    return sbmod


def _rel(got: dict, ref: so.BS) -> float:
    rb = ref.blocks_by_key()
    assert set(got) == set(rb)
    scale = max(np.max(np.abs(v)) for v in rb.values())
    return max(np.max(np.abs(got[k] - v)) for k, v in rb.items()) / scale


def _problem(sb, n, chi, seed):
    return pxp.PxpProblem(n, chi, seed, ctx=sb.Context(0))


@pytest.fixture(scope="module", params=[(12, 16, 5), (64, 256, 64)], ids=["n12_chi16", "n64_chi256"])
def pair(request, sb):
    n, chi, seed = request.param
    return _problem(sb, n, chi, seed), pr.OracleProblem(n, chi, seed)


def test_environments(pair):
    dev, ora = pair
    for got, ref in ((dev.L, ora.L), (dev.R, ora.R)):
        assert got.dims == ref.dims and got.keys == ref.keys
        assert _rel(got.blocks_by_key(), ref) <= FP64_RTOL


def test_heff_fp64(pair):
    dev, ora = pair
    out, ref = dev.apply(dev.psi), ora.apply(ora.psi)
    assert out.dims == ref.dims and out.keys == ref.keys
    assert _rel(out.blocks_by_key(), ref) <= FP64_RTOL


def test_heff_intermediates_follow_oracle(pair):
    """Every intermediate of the matvec has the oracle's keys; the COO steps
    (T2, T3 from the device's own T1) are scaled adds with exact 0/1 factors."""
    dev, ora = pair
    t = dev._run(pxp.HEFF_STEPS, {"psi": dev.psi, "L": dev.L, "R": dev.R, "W1f": dev.Wf, "W2f": dev.Wf})
    r = pr.o_run(pxp.HEFF_STEPS, {"psi": ora.psi, "L": ora.L, "R": ora.R, "W1f": ora.Wf, "W2f": ora.Wf})
    for name in ("T1", "T1f", "T2", "T2f", "T3", "T4"):
        assert t[name].keys == r[name].keys, name
    # the oracle's COO step on the device's T1f: bit for bit
    t1f = pr.o_bs(t["T1f"].dims, t["T1f"].keys, t["T1f"].data)
    t2 = pr.o_contract(list(pxp.HEFF_STEPS[2][2]), 2, ora.Wf, list(pxp.LABELS["W1f"]), t1f,
                       ["qlp", "s2", "qr", "x1", "lp", "r"])
    gb = t["T2"].blocks_by_key()
    for k, v in t2.blocks_by_key().items():
        assert np.array_equal(gb[k], v), k


def test_heff_tf32x3(pair):
    """The matvec with the dense contractions in 3xTF32 on the tensor cores
    (FP32 accumulation), on the FP64 environments."""
    dev, ora = pair
    dev.ctx.set_precision("tf32x3")
    try:
        out = dev.apply(dev.psi)
    finally:
        dev.ctx.set_precision("f64")
    ref = ora.apply(ora.psi)
    assert out.keys == ref.keys
    err = _rel(out.blocks_by_key(), ref)
    assert err <= TF32X3_RTOL, err
    if dev.chi > 16:
        # the tensor-core path ran (FP64 agrees to about 1e-15); blocks with 16
        # or fewer rows or columns take the FP64 thin-block kernel in every
        # precision
        assert err > 1e-11


def test_heff_symmetric(sb, pair):
    dev, _ = pair
    rng = np.random.Generator(np.random.PCG64(11))
    phi_h = rng.standard_normal(dev.psi_host.shape)
    phi = dev._bs(*pxp.psi_blocks(phi_h))
    a = sb.dot(phi, dev.apply(dev.psi))
    b = sb.dot(dev.apply(phi), dev.psi)
    assert abs(a - b) <= 1e-12 * max(abs(a), 1.0)


def test_mpo_apply_every_site(pair):
    """MPO x MPS (COO x block-sparse, contract_prefix!) on every site tensor
    of the chain: bit for bit against the oracle."""
    dev, ora = pair
    lab_c = ["sp", "wl", "wr", "ql", "qr", "l", "r"]
    for k, A in enumerate(dev.sites):
        if A is None:
            continue
        out = dev.apply_mpo(dev._bs(*pxp.site_blocks(A)))
        Ao = pr.o_bs(*pxp.site_blocks(A))
        dims = (pxp.D, pxp.W, pxp.W, 1, 1) + A.shape[::2]
        ref = so.contract(so.BS.empty(dims, 2), lab_c, ora.Wc, ["sp", "s", "wl", "wr"], Ao,
                          ["ql", "s", "qr", "l", "r"])
        assert out.keys == ref.keys, k
        gb = out.blocks_by_key()
        for key, v in ref.blocks_by_key().items():
            assert np.array_equal(gb[key], v), (k, key)


@pytest.mark.parametrize("precision", ["f64", "tf32x3"])
def test_heff_graph_replay(sb, pair, precision):
    """The matvec captured as one CUDA graph: a replay after psi changes in
    place equals the eager matvec of the new psi, bit for bit."""
    dev, _ = pair
    dev.ctx.set_precision(precision)
    try:
        psi = dev._bs(*pxp.psi_blocks(dev.psi_host))
        graph, out = dev.capture(psi)
        sb.scale_(psi, -0.5)
        graph.launch()
        got = out.blocks_by_key()
        want = dev.apply(psi).blocks_by_key()
    finally:
        dev.ctx.set_precision("f64")
    assert set(got) == set(want)
    for k, v in want.items():
        assert np.array_equal(got[k], v), k


def test_heff_aliased(sb, pair):
    """The aliased form of the matvec (W as templates I, P, X; dense psi and
    environments): same template structure as the oracle, the same H_eff . psi
    as the oracle and as the COO form, to 1e-13."""
    dev, ora = pair
    ops = dev.aliased_operands()
    psi_d = sb.DenseTensor(dev.psi_host, ctx=dev.ctx)
    got = dev.apply_aliased(psi_d, ops)
    ref = ora.apply_aliased(ora.psi_host)
    assert got.keys == ref.keys == [()]
    assert got.n_templates == ref.n_templates
    g, r = got.logical_blocks()[()], ref.logical_blocks()[()]
    assert np.max(np.abs(g - r)) <= FP64_RTOL * np.max(np.abs(r))
    coo = pxp.psi_from_blocks(*_keys_data(dev.apply(dev.psi)), dev.psi.dims)
    assert np.max(np.abs(g.reshape(coo.shape, order="F") - coo)) <= FP64_RTOL * np.max(np.abs(coo))


def _keys_data(T):
    b = T.blocks_by_key()
    keys = sorted(b, key=lambda k: tuple(reversed(k)))
    return keys, np.concatenate([b[k] for k in keys])
