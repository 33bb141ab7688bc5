"""The second association of the two-site H_eff chain on the device:
W12 = W1·W2 (MPO blocks only), then ψ·L, ·W12, ·R (``HeffChain(w12=True)``).

* W12 on the device has the oracle's key list (bit-exact) and blocks within
  1e-12, for ragged and zero-padded MPO tensors;
* H_eff·ψ through the W12 chain matches the oracle's four-step chain (the
  reference's order) within 1e-12 per block, ragged and padded;
* it replays from a CUDA graph to the same bits as the eager chain, and the
  Lanczos eigensolver on it finds the same lowest Ritz value (1e-12);
* at the chi = 2048 benchmark size it agrees with the four-step chain within
  1e-12 and repeated applies are bit-identical.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from tests.heff_dense import small_layout

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _setup(ragged, seed, chi=24):
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    lay = small_layout(chi)
    rng = np.random.Generator(np.random.PCG64(seed))
    ops = qn.hermitian_operators(lay, rng)
    ops["psi"] = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    ctx = sb.Context(0)
    dev, pad = {}, {}
    for n, (k, d, e) in ops.items():
        pad[n] = (k, qn.pad_ragged(lay, n, k, d, e))
        if ragged:
            dev[n] = sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx, block_dims=e)
        else:
            dev[n] = sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, pad[n][1], ctx=ctx)
    orc = {n: so.BS(lay.dims[n], lay.n2[n], k, list(range(1, len(k) + 1)), d) for n, (k, d) in pad.items()}
    return sb, qn, lay, ctx, dev, orc


def _uniform_blocks(sb, t):
    u = sb.to_uniform(t) if t.is_ragged else t
    return u.keys, u.blocks_by_key()


@pytest.mark.parametrize("ragged", [True, False])
def test_w12_and_chain_match_oracle(ragged):
    sb, qn, lay, ctx, dev, orc = _setup(ragged, seed=5)
    lab = lay.labels
    chain = qn.HeffChain(lay, ctx, w12=True)
    out = chain.apply(dev["psi"], dev["L"], dev["W1"], dev["W2"], dev["R"])
    # W12 itself
    w12 = so.contract(so.BS.empty(lay.dims["W12"], 2), lab["W12"], orc["W1"], lab["W1"], orc["W2"], lab["W2"])
    keys, blocks = _uniform_blocks(sb, chain.out["W12"])
    assert keys == w12.keys
    ref = w12.blocks_by_key()
    for k in ref:
        assert _rel(blocks[k], ref[k]) <= RTOL
    # the matvec against the oracle's four-step chain
    t = dict(orc)
    for c, a, b in qn.HeffChain.STEPS:
        t[c] = so.contract(so.BS.empty(lay.dims[c], lay.n2[c]), lab[c], t[a], lab[a], t[b], lab[b])
    keys, blocks = _uniform_blocks(sb, out)
    assert keys == t["T4"].keys
    ref = t["T4"].blocks_by_key()
    for k in ref:
        assert _rel(blocks[k], ref[k]) <= RTOL


def test_w12_graph_replay_and_lanczos():
    sb, qn, lay, ctx, dev, orc = _setup(True, seed=6)
    from sparsebackends_b200 import krylov
    ops = (dev["L"], dev["W1"], dev["W2"], dev["R"])
    eager = qn.HeffChain(lay, ctx, w12=True)
    want = eager.apply(dev["psi"], *ops).data
    chain = qn.HeffChain(lay, ctx, w12=True)
    g = chain.capture(dev["psi"], *ops)
    sb.fill_(chain.out["T4"], 0.0)
    g.launch()
    assert np.array_equal(chain.out["T4"].data, want)
    op4 = qn.HeffOperator(lay, *ops, ctx)
    op3 = qn.HeffOperator(lay, *ops, ctx, w12=True)
    v4, _, _ = krylov.eigsolve(op4, dev["psi"], 1, "SR", krylovdim=6, maxiter=2, tol=1e-14)
    v3, _, _ = krylov.eigsolve(op3, dev["psi"], 1, "SR", krylovdim=6, maxiter=2, tol=1e-14)
    assert abs(v3[0] - v4[0]) <= 1e-12 * abs(v4[0])


def test_w12_full_size_agrees_with_four_step_chain():
    import bench
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    lay = bench.workload(2048)
    _, host_r = bench.host_tensors(lay, 2026, with_ragged=True)
    ctx = sb.Context(0)
    dev = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx, block_dims=e)
           for n, (k, d, e) in host_r.items()}
    args = (dev["psi"], dev["L"], dev["W1"], dev["W2"], dev["R"])
    four = qn.HeffChain(lay, ctx).apply(*args)
    k4, d4 = four.keys, np.array(four.data, copy=True)
    chain = qn.HeffChain(lay, ctx, w12=True)
    out = chain.apply(*args)
    assert out.keys == k4 and out.block_dims == four.block_dims
    d3 = np.array(out.data, copy=True)
    assert _rel(d3, d4) <= RTOL
    assert np.array_equal(chain.apply(*args).data, d3)
