"""The two merge-join orders of contract_shared! (``oracle.join_order``).

The reference's ``_cmp_join_tuple`` (contract_bs_bs.jl:430-442) compares the
join tuple from its first axis while ``permutedims`` sorts keys column-major
with the join axes last (storage.jl:188-266, contract_bs_bs.jl:513-566), so the
last join axis is the most significant.  With two or more join axes whose value
sets differ between the operands, the reference's merge advances past runs
that still hold matches.  The oracle's default order compares from the last
join axis down, consistent with the sort; ``join_order("reference")`` runs the
reference's comparison unchanged.

Enumerated here:

* every known-answer case restated from the reference's tests: both orders give
  bit-identical results (the reference's own tests cannot tell them apart);
* the chain and environment contractions of the N = 16 centre problem and of the
  J1-J2 6x6-sized problem (``tests/join_cases.py``): the list of contractions
  where the reference's order loses matched pairs is pinned below, and on
  each of them the default order equals the dense einsum of the operands.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from tests import join_cases as jc
from tests import kat_cases as kc
from tests.test_oracle_kat import make_operand

# contraction -> output keys the reference's order drops (on all four it loses
# matched pairs, so block values differ as well)
DIVERGENT = {
    "n16:chain_w12:T3=T1*W12": 0,
    "n16:make_R(site 9):F2=F1*W": 5,
    "n16:make_L(site 1, boundary):E2=E1*W": 2,
    "j1j2:make_L:L'=E2*A": 0,
}


def _cases():
    return jc.centre_problem_cases() + jc.j1j2_sized_cases()


@pytest.fixture(scope="module")
def workload_cases():
    return _cases()


def test_known_answer_cases_agree():
    n = 0
    for c in kc.all_cases():
        if c.expect_error or c.kind_C != "bs":
            continue
        A, B = make_operand(c.kind_A, c.A, c.n2A), make_operand(c.kind_B, c.B, c.n2B)
        got = so.contract(so.BS.empty(c.dimsC, c.n2C), c.labelsC, A, c.labelsA, B, c.labelsB)
        with so.join_order("reference"):
            ref = so.contract(so.BS.empty(c.dimsC, c.n2C), c.labelsC, A, c.labelsA, B, c.labelsB)
        assert got.keys == ref.keys and np.array_equal(got.data, ref.data), c.name
        n += 1
    assert n > 100


def test_workload_divergence_list(workload_cases):
    found = {}
    for name, C0, lc, A, la, B, lb in workload_cases:
        r = jc.compare_join_orders(C0, lc, A, la, B, lb)
        if r["same_keys"] and r["max_rel_diff"] == 0.0:
            continue
        assert r["njoin"] >= 2, name  # one join axis: the two orders are the same comparison
        assert r["extra"] == 0, name  # the reference's order only loses pairs
        found[name] = r["missing"]
    assert found == DIVERGENT


@pytest.mark.parametrize("name", sorted(DIVERGENT))
def test_default_order_matches_dense(workload_cases, name):
    (_, C0, lc, A, la, B, lb), = [c for c in workload_cases if c[0] == name]
    got = so.contract(so.BS.empty(C0.dims, C0.n2), lc, A, la, B, lb)
    want = kc.dense_contract(so.bs_to_dense(A), la, so.bs_to_dense(B), lb, lc)
    assert np.abs(so.bs_to_dense(got) - want).max() <= 1e-12 * max(np.abs(want).max(), 1.0)
    with so.join_order("reference"):
        ref = so.contract(so.BS.empty(C0.dims, C0.n2), lc, A, la, B, lb)
    assert np.abs(so.bs_to_dense(ref) - want).max() > 1e-6 * np.abs(want).max()


def test_join_order_restores():
    assert so.JOIN_ORDER == "sorted"
    with so.join_order("reference"):
        assert so.JOIN_ORDER == "reference"
    assert so.JOIN_ORDER == "sorted"
    with pytest.raises(so.OracleError):
        so.join_order("lexicographic")
