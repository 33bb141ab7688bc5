"""The library's device matcher on the chain and environment contractions of
``tests/join_cases.py``, including the ones where the reference's merge order
loses matched pairs: output keys identical to the oracle's (default, sort-
consistent order), every block to 1e-12 relative Frobenius error."""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from tests import join_cases as jc

pytestmark = pytest.mark.gpu

CASES = jc.centre_problem_cases() + jc.j1j2_sized_cases()


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as m
    return m


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_device_matches_oracle(sb, case):
    name, C0, lc, A, la, B, lb = case
    ctx = sb.default_context()
    ref = so.contract(so.BS.empty(C0.dims, C0.n2), lc, A, la, B, lb)
    C = sb.NewBlockSparseSorted.empty(C0.dims, C0.n2, ctx=ctx)
    sb.contract_(C, lc, sb.NewBlockSparseSorted(A.dims, A.n2, A.keys, A.ids, A.data, ctx=ctx), la,
                 sb.NewBlockSparseSorted(B.dims, B.n2, B.keys, B.ids, B.data, ctx=ctx), lb)
    assert C.keys == ref.keys
    gb = C.blocks_by_key()
    for k, v in ref.blocks_by_key().items():
        assert np.linalg.norm(np.asarray(gb[k]) - v) <= 1e-12 * max(np.linalg.norm(v), 1e-300), k
