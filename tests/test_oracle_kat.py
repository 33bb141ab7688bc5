"""Pin the CPU oracle to the reference's own known-answer tests.

Every case here is restated from ``SparseBackends/test/**`` (file:line in the
case name / docstring).  The oracle must reproduce the reference's exact key
lists and exact block values on these small dyadic inputs.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from tests import kat_cases as kc


def make_operand(kind, arr, n2):
    if kind == "bs":
        return so.blocksparse_from_dense(arr, n2, atol=0.0, rtol=0.0)
    if kind == "coo":
        return so.coo_from_dense(arr, atol=0.0, rtol=0.0)
    return arr


def run_oracle(case: kc.Case):
    A = make_operand(case.kind_A, case.A, case.n2A)
    B = make_operand(case.kind_B, case.B, case.n2B)
    if case.kind_C == "bs":
        C = so.BS.empty(case.dimsC, case.n2C)
    else:
        C = so.COO(case.dimsC)
    return so.contract(C, case.labelsC, A, case.labelsA, B, case.labelsB)


@pytest.mark.parametrize("case", kc.all_cases(), ids=lambda c: c.name)
def test_oracle_matches_reference_kat(case):
    if case.expect_error:
        with pytest.raises(so.OracleError):
            run_oracle(case)
        return
    C = run_oracle(case)
    ref = case.C_dense
    if case.kind_C == "bs":
        Cref = so.blocksparse_from_dense(ref, case.n2C, atol=0.0, rtol=0.0)
        assert C.dims == Cref.dims
        assert C.blksize == Cref.blksize
        assert C.keys == Cref.keys
        dC, dR = C.blocks_by_key(), Cref.blocks_by_key()
        for k in dR:
            assert np.array_equal(dC[k], dR[k]), k
    else:
        so.coo_sort(C)
        Cref = so.coo_from_dense(ref, atol=0.0, rtol=0.0)
        assert C.keys == Cref.keys
        assert C.vals == Cref.vals


def test_coo_dense_zero_slice_follows_code():
    """coo_dense.jl:163-189 expects no blocks, but the code creates a block for
    every in-range nnz (contract_coo_dense.jl:113-122). The oracle follows the code."""
    A = np.zeros((3, 4)); A[1, 2] = 1.0
    B = np.zeros((5, 4))
    C = so.BS.empty((3, 5), 1)
    so.contract(C, ["i", "x"], so.coo_from_dense(A, atol=0.0), ["i", "r"], B, ["x", "r"])
    assert C.keys == [(2,)]
    assert np.all(C.block(C.ids[0]) == 0)


# ── storage known answers ────────────────────────────────────────────────


def test_coo_2d_keys():
    """test/coo/test.jl:10-24."""
    A = np.zeros((4, 3)); A[2, 0] = 2.0; A[0, 1] = -5.0; A[3, 2] = 7.0
    S = so.coo_from_dense(A, atol=0.0)
    assert np.array_equal(so.coo_to_dense(S), A)
    assert S.keys == [(3, 1), (1, 2), (4, 3)]
    assert S.vals == [2.0, -5.0, 7.0]


def test_coo_4d_keys():
    """test/coo/test.jl:26-39."""
    A = np.zeros((2, 2, 2, 3))
    A[1, 0, 0, 0] = 11.0; A[0, 1, 1, 0] = -3.0; A[1, 1, 0, 1] = 5.0; A[0, 0, 1, 2] = 7.0
    S = so.coo_from_dense(A, atol=0.0)
    assert S.keys == [(2, 1, 1, 1), (1, 2, 2, 1), (2, 2, 1, 2), (1, 1, 2, 3)]


def test_coo_permutedims_keys():
    """test/coo/test.jl:64-81."""
    A = np.zeros((3, 2, 4)); A[0, 0, 0] = 1.0; A[2, 1, 3] = -2.0; A[1, 0, 2] = 7.0
    S = so.coo_from_dense(A, atol=0.0)
    Sp = so.coo_sort(so.coo_permutedims(S, [3, 1, 2]))
    assert Sp.keys == [(1, 1, 1), (3, 2, 1), (4, 3, 2)]
    assert np.array_equal(so.coo_to_dense(Sp), np.transpose(A, (2, 0, 1)))


def _storage_tensor():
    dims = (4, 3, 2, 5)
    A = np.zeros(dims)
    for k in range(2):
        for l in range(5):
            A[0, 1, k, l] = 10 + k * 5 + (l + 1)
            A[2, 0, k, l] = -(k * 5 + (l + 1))
    A[3, 2, 0, 0] = 7
    A[3, 2, 1, 4] = -9
    return A


def test_bs_from_dense_keys_and_roundtrip():
    """test/blocksparse/test_convertor.jl:6-44 and test_storage.jl:56-73."""
    A = np.zeros((6, 5)); A[1, :] = (1, 0, 2, 0, 3); A[4, :] = (-1, 4, 0, 0, 7)
    B = so.blocksparse_from_dense(A, 1)
    assert np.array_equal(so.bs_to_dense(B), A)
    assert B.blksize == 5 and B.keys == [(2,), (5,)] and len(B.data) == 10
    D = _storage_tensor()
    B = so.blocksparse_from_dense(D, 2)
    assert np.array_equal(so.bs_to_dense(B), D)
    assert B.blksize == 10 and B.keys == [(3, 1), (1, 2), (4, 3)]


def test_bs_getindex_setindex():
    """test/blocksparse/test_storage.jl:8-54."""
    A = so.BS.empty((4, 3, 2, 5), 2)
    assert A.getindex(1, 1, 1, 1) == 0.0
    A.setindex(7.5, 3, 1, 2, 5)
    A.setindex(-2.0, 3, 1, 1, 1)
    A.setindex(3.0, 1, 2, 1, 1)
    assert A.getindex(3, 1, 2, 5) == 7.5
    assert A.getindex(3, 1, 1, 1) == -2.0
    assert A.getindex(1, 2, 1, 1) == 3.0
    assert A.getindex(4, 3, 1, 1) == 0.0
    assert A.keys == [(3, 1), (1, 2)]
    assert len(A.data) == len(A.keys) * A.blksize


@pytest.mark.parametrize("perm", [[2, 1, 3, 4], [1, 2, 4, 3], [2, 1, 4, 3]])
def test_bs_permutedims(perm):
    """test/blocksparse/test_storage.jl:75-100."""
    D = _storage_tensor()
    A = so.blocksparse_from_dense(D, 2)
    B = so.bs_permutedims(A, perm)
    assert np.array_equal(so.bs_to_dense(B), np.transpose(D, [p - 1 for p in perm]))


def test_bs_permutedims_rejects_cross():
    """test/blocksparse/test_storage.jl:102-111."""
    D = np.zeros((4, 3, 2, 5)); D[0, 1, 0, 0] = 1.0
    A = so.blocksparse_from_dense(D, 2)
    with pytest.raises(so.OracleError):
        so.bs_permutedims(A, [3, 2, 1, 4])


# ── Kahan precision study (test_kernel_precision.jl:207-414) ─────────────


@pytest.mark.parametrize("seed,left,rl,da,b,scale", [(42, 4, 3, 4, 3, 1.0), (77, 8, 8, 6, 6, 50.0), (99, 8, 8, 6, 6, 20.0)])
def test_prefix_outer_bd_kahan_precision(seed, left, rl, da, b, scale):
    """Kahan-compensated prefix_outer_bd vs an exact (fsum) triple loop.

    Julia's MersenneTwister streams cannot be reproduced; the shapes, seeds
    and scales of test_kernel_precision.jl are kept with numpy's PCG64."""
    import math
    rng = np.random.Generator(np.random.PCG64(seed))
    A = rng.standard_normal((left, rl, da)) * scale
    B = rng.standard_normal((rl, b))
    Abs = so.blocksparse_from_dense(A, 1)
    C = so.BS.empty((left, da, b), 2)
    so.contract(C, ["left", "da", "b"], Abs, ["left", "rlab", "da"], B, ["rlab", "b"])
    got = so.bs_to_dense(C)
    exact = np.zeros((left, da, b))
    for i in range(left):
        for x in range(da):
            for y in range(b):
                exact[i, x, y] = math.fsum(A[i, r, x] * B[r, y] for r in range(rl))
    err = np.linalg.norm(got - exact)
    assert err <= 4 * np.finfo(float).eps * np.linalg.norm(exact) + 1e-300


# ── aliased kernels agree with the materialised block-sparse kernels ─────


def _aliased_from_dense(arr, n2):
    return so.aliased_from_blocksparse_unique(so.blocksparse_from_dense(arr, n2))


def _check_aliased_equals_bs(Cal, Cbs):
    Cal_bs = so.aliased_to_blocksparse(Cal)
    assert Cal_bs.keys == Cbs.keys
    dA, dB = Cal_bs.blocks_by_key(), Cbs.blocks_by_key()
    for k in dB:
        np.testing.assert_allclose(dA[k], dB[k], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("case", kc.bs_dense_cases()[:4] + kc.bs_bs_prefix_cases()[:4]
                         + kc.bs_bs_multi_cases()[:3], ids=lambda c: c.name)
def test_aliased_matches_blocksparse(case):
    A = _aliased_from_dense(case.A, case.n2A)
    B = case.B if case.kind_B == "dense" else _aliased_from_dense(case.B, case.n2B)
    Cal = so.contract(so.Aliased.empty(case.dimsC, case.n2C), case.labelsC, A, case.labelsA, B, case.labelsB)
    Cbs = run_oracle(case)
    # Aliased kernels create blocks for every contribution; the reference BS
    # kernels too (structural rules), so the key lists agree.
    _check_aliased_equals_bs(Cal, Cbs)


def test_aliased_coo_dense_demotion():
    """contract_aliased_coo_dense.jl:92-138: same-ckey contributions demote."""
    A = np.zeros((3, 4)); A[0, 0] = 2.0; A[0, 1] = -1.0; A[2, 1] = 0.5; A[1, 3] = 3.0
    B = np.zeros((5, 4)); B[1, 0] = 7.0; B[4, 1] = -2.0; B[0, 3] = 1.0; B[2, 1] = 4.0
    Acoo = so.coo_from_dense(A, atol=0.0)
    Cal = so.contract(so.Aliased.empty((3, 5), 1), ["i", "x"], Acoo, ["i", "r"], B, ["x", "r"])
    Cbs = so.contract(so.BS.empty((3, 5), 1), ["i", "x"], Acoo, ["i", "r"], B, ["x", "r"])
    _check_aliased_equals_bs(Cal, Cbs)
    # key (1,) got rv=1 and rv=2 → demoted to its own template with scalar 1
    i = Cal.keys.index((1,))
    assert Cal.scalars[i] == 1.0
    # keys (3,) and its rv=2 template is shared with nobody else but stays aliased
    j = Cal.keys.index((3,))
    assert Cal.scalars[j] == 0.5


def test_bs_is_dense():
    """is_dense (src/blocksparse/storage.jl:413-425): every prefix combination has a block."""
    full = so.blocksparse_from_dense(np.arange(1.0, 25.0).reshape(2, 3, 4), 1)
    assert so.bs_is_dense(full)
    A = np.zeros((2, 3, 4))
    A[0, 1] = 1.0
    assert not so.bs_is_dense(so.blocksparse_from_dense(A, 1))
    assert so.bs_is_dense(so.blocksparse_from_dense(np.ones((3, 4)), 2))  # no prefix
