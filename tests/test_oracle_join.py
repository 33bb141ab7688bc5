"""contract_shared! with two shared prefix labels whose value sets differ
between the operands (the first MPS environment update of an MPO chain has
this shape: the boundary environment holds one MPO channel sector, the MPO
tensor all of them).

The reference's merge-join compares join tuples first-axis-major while its
keys are sorted last-axis-major, so in this case it loses matched pairs; the
oracle and the library compare in the sort order.  Checked against the dense
einsum, which is what contract! computes by definition."""
import numpy as np

from oracle import sparse_oracle as so


def test_two_label_join_with_unequal_tuple_sets():
    rng = np.random.Generator(np.random.PCG64(3))
    # A[(p, w, s) | m] has w = 2 only; B[(w, s, t) | n] has w in 1..3
    Ad = np.zeros((2, 3, 2, 4))
    Ad[:, 1] = rng.standard_normal((2, 2, 4))
    Bd = rng.standard_normal((3, 2, 3, 5))  # every (w, s) present, including (3, 1)
    A, B = so.blocksparse_from_dense(Ad, 1), so.blocksparse_from_dense(Bd, 1)
    C = so.contract(so.BS.empty((2, 3, 4, 5), 2), ["p", "t", "m", "n"], A, ["p", "w", "s", "m"], B,
                    ["w", "s", "t", "n"])
    want = np.einsum("pwsm,wstn->ptmn", Ad, Bd)
    assert np.allclose(so.bs_to_dense(C), want, atol=1e-13)
