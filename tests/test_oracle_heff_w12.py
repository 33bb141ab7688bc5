"""CPU checks of the second association of the two-site H_eff chain.

ITensorMPS applies H_eff as ((ψ·L)·W1)·W2)·R.  The library also offers
ψ·L·(W1·W2)·R: the two MPO tensors contracted with each other first (W12, a
contraction of MPO blocks only), then three contractions.  On the oracle:

* the key simulation of both orders gives the same output key list, and the
  W12 order does no more algorithmic FLOPs;
* both orders give the same H_eff·ψ (1e-12 relative per block) on the
  reference's zero-padded layout.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from sparsebackends_b200 import qn
from tests.heff_dense import small_layout


def _keys_of_output(lay, steps):
    st = qn.chain_structure(lay, steps)[-1]
    lc = lay.labels["T4"]
    pc = len(lc) - lay.n2["T4"]
    return {tuple(kv[x] for x in lc[:pc]) for kv in st["pairs"]}


@pytest.mark.parametrize("chi", [24, 64])
def test_same_output_structure_and_no_more_flops(chi):
    lay = small_layout(chi)
    assert _keys_of_output(lay, qn.HeffChain.STEPS) == _keys_of_output(lay, qn.HeffChain.STEPS_W12)
    f4 = qn.chain_flops(lay, padded=False, steps=qn.HeffChain.STEPS)
    f3 = qn.chain_flops(lay, padded=False, steps=qn.HeffChain.STEPS_W12)
    assert f3 <= f4


def _run(lay, t, steps):
    t = dict(t)
    lab = lay.labels
    for c, a, b in steps:
        t[c] = so.contract(so.BS.empty(lay.dims[c], lay.n2[c]), lab[c], t[a], lab[a], t[b], lab[b])
    return t["T4"]


@pytest.mark.parametrize("seed", [0, 1])
def test_both_orders_give_the_same_matvec(seed):
    lay = small_layout(24)
    rng = np.random.Generator(np.random.PCG64(seed))
    t = {}
    for name in ("psi", "L", "W1", "W2", "R"):
        keys, data = qn.random_block_tensor(lay, name, rng, 0.5)
        t[name] = so.BS(lay.dims[name], lay.n2[name], keys, list(range(1, len(keys) + 1)), data)
    a = _run(lay, t, qn.HeffChain.STEPS)
    b = _run(lay, t, qn.HeffChain.STEPS_W12)
    assert a.keys == b.keys
    ab, bb = a.blocks_by_key(), b.blocks_by_key()
    for k in ab:
        n = np.linalg.norm(ab[k])
        assert np.linalg.norm(ab[k] - bb[k]) <= 1e-12 * max(n, 1e-300)
