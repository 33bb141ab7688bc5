"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle.

Bar (per the reference semantics):
* key lists / block structure: bit-exact, including value-dependent rules;
* values: bit-exact for the hand-loop kernels the reference writes elementwise
  (outer products, Kahan sums, COO axpys); ≤ 1e-12 relative Frobenius error per
  block for the BLAS (GEMM/ger) kernels, which the reference delegates to
  OpenBLAS with an unspecified summation order.
"""
import itertools

import numpy as np
import pytest

from oracle import sparse_oracle as so
from tests import kat_cases as kc

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as sbmod
    return sbmod


def lib_operand(sb, x):
    if isinstance(x, so.BS):
        return sb.NewBlockSparseSorted(x.dims, x.n2, x.keys, x.ids, x.data)
    if isinstance(x, so.COO):
        return sb.COOTensor(x.dims, x.keys, x.vals, x.dirty)
    if isinstance(x, so.Aliased):
        return sb.AliasedBlockSparse(x.dims, x.n2, x.templates, x.keys, x.alias_ids, x.scalars)
    return sb.DenseTensor(np.asarray(x))


def lib_empty_like(sb, C):
    if isinstance(C, so.BS):
        return sb.NewBlockSparseSorted.empty(C.dims, C.n2)
    if isinstance(C, so.COO):
        return sb.COOTensor(C.dims)
    return sb.AliasedBlockSparse.empty(C.dims, C.n2)


def rel_err(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def assert_bs_equal(got, ref: so.BS, exact=False):
    assert got.dims == ref.dims
    assert got.blksize == ref.blksize
    assert got.keys == ref.keys
    gb, rb = got.blocks_by_key(), ref.blocks_by_key()
    for k, v in rb.items():
        if exact:
            assert np.array_equal(gb[k], v), k
        else:
            assert rel_err(gb[k], v) <= RTOL, (k, rel_err(gb[k], v))


def assert_aliased_equal(got, ref: so.Aliased):
    assert got.keys == ref.keys
    gb, rb = got.logical_blocks(), ref.logical_blocks()
    for k, v in rb.items():
        assert rel_err(gb[k], v) <= RTOL, k


def run_both(sb, C0, lC, A, lA, B, lB):
    """Run the oracle and the library on identical operands."""
    Cref = so.contract(C0, lC, A, lA, B, lB)
    Cg = lib_empty_like(sb, C0)
    sb.contract_(Cg, lC, lib_operand(sb, A), lA, lib_operand(sb, B), lB)
    return Cg, Cref


# ── the reference's known-answer cases ───────────────────────────────────


def _make(kind, arr, n2):
    if kind == "bs":
        return so.blocksparse_from_dense(arr, n2)
    if kind == "coo":
        return so.coo_from_dense(arr, atol=0.0)
    return arr


EXACT_FAMILIES = ("bs_bs_prefix", "bs_dense", "coo_bs", "coo_dense", "coo_coo")


@pytest.mark.parametrize("case", kc.all_cases(), ids=lambda c: c.name)
def test_kat_parity(sb, case):
    A = _make(case.kind_A, case.A, case.n2A)
    B = _make(case.kind_B, case.B, case.n2B)
    C0 = so.BS.empty(case.dimsC, case.n2C) if case.kind_C == "bs" else so.COO(case.dimsC)
    if case.expect_error:
        with pytest.raises(sb.SparseBackendsError) as ei:
            Cg = lib_empty_like(sb, C0)
            sb.contract_(Cg, case.labelsC, lib_operand(sb, A), case.labelsA, lib_operand(sb, B), case.labelsB)
        assert ei.value.status == "SB_ERR_UNSUPPORTED_LAYOUT"
        return
    Cg, Cref = run_both(sb, C0, case.labelsC, A, case.labelsA, B, case.labelsB)
    if case.kind_C == "bs":
        # dyadic inputs: every kernel must match the reference's exact answer
        assert_bs_equal(Cg, Cref, exact=True)
        Cdense = so.blocksparse_from_dense(case.C_dense, case.n2C)
        assert_bs_equal(Cg, Cdense, exact=True)
    else:
        Cg_sorted = sb.sort_(Cg)
        so.coo_sort(Cref)
        assert Cg_sorted.keys == Cref.keys
        assert Cg_sorted.vals == Cref.vals


# ── seeded random cases, larger than the KATs ────────────────────────────


def rand_bs(rng, dims, n2, density=0.5, scale=1.0):
    P = len(dims) - n2
    A = rng.standard_normal(dims) * scale
    pdims = dims[:P]
    mask = rng.random(pdims) < density
    A = A * mask.reshape(pdims + (1,) * n2)
    return A, so.blocksparse_from_dense(A, n2)


def rand_coo(rng, dims, density=0.3):
    A = rng.standard_normal(dims) * (rng.random(dims) < density)
    return A, so.coo_from_dense(A, atol=0.0)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_shared_bb(sb, seed):
    """contract_shared! BS×BS (contract_bs_bs.jl:572-730) with join + GEMM."""
    rng = np.random.Generator(np.random.PCG64(seed))
    # A[(i, q) | (m, k)] x B[(q, j) | (k, n)] -> C[(i, j) | (m, n)]
    I, Q, J, M, K, N = 3, 4, 3, 17, 23, 9
    _, A = rand_bs(rng, (I, Q, M, K), 2)
    _, B = rand_bs(rng, (Q, J, K, N), 2)
    for lC in (["i", "j", "m", "n"], ["j", "i", "n", "m"]):
        Cg, Cref = run_both(sb, so.BS.empty(tuple({"i": I, "j": J, "m": M, "n": N}[l] for l in lC), 2), lC,
                            A, ["i", "q", "m", "k"], B, ["q", "j", "k", "n"])
        assert_bs_equal(Cg, Cref)


@pytest.mark.parametrize("seed", [4, 5])
def test_random_shared_bb_permuted_operands(sb, seed):
    """Forces block-tail permutes and key re-sorting on both operands."""
    rng = np.random.Generator(np.random.PCG64(seed))
    _, A = rand_bs(rng, (5, 3, 7, 33, 40), 2)   # (q, i, m | k, x)
    _, B = rand_bs(rng, (4, 5, 33, 6), 2)       # (j, q | k, n)
    lA, lB = ["q", "i", "m", "k", "x"], ["j", "q", "k", "n"]
    lC = ["m", "j", "i", "x", "n"]
    Cg, Cref = run_both(sb, so.BS.empty((7, 4, 3, 40, 6), 2), lC, A, lA, B, lB)
    assert_bs_equal(Cg, Cref)


@pytest.mark.parametrize("seed", [6, 7])
def test_random_shared_bd(sb, seed):
    """contract_shared! BS×Dense (contract_bs_dense.jl:411-619): the H_eff workhorse."""
    rng = np.random.Generator(np.random.PCG64(seed))
    # W[(s', s) | (wl, wr)] x T(s, wl, x, y) -> C[(s') | (wr, x, y)]
    d, w, X, Y = 2, 7, 19, 11
    _, W = rand_bs(rng, (d, d, w, w), 2, density=0.8)
    T = rng.standard_normal((d, w, X, Y))
    for lC in (["sp", "wr", "x", "y"], ["sp", "x", "y", "wr"]):
        dims = tuple({"sp": d, "wr": w, "x": X, "y": Y}[l] for l in lC)
        Cg, Cref = run_both(sb, so.BS.empty(dims, 3), lC, W, ["sp", "s", "wl", "wr"], T, ["s", "wl", "x", "y"])
        assert_bs_equal(Cg, Cref)


@pytest.mark.parametrize("seed", [8, 9])
def test_random_prefix_outer_bd_kahan_bit_exact(sb, seed):
    """contract_prefix_outer_bd! with Kahan sums is reproduced bit for bit."""
    rng = np.random.Generator(np.random.PCG64(seed))
    _, A = rand_bs(rng, (6, 8, 5), 1, density=0.9, scale=50.0)  # (left, r | da)
    B = rng.standard_normal((8, 7))                             # (r, b)
    Cg, Cref = run_both(sb, so.BS.empty((6, 5, 7), 2), ["left", "da", "b"], A, ["left", "r", "da"], B, ["r", "b"])
    assert_bs_equal(Cg, Cref, exact=True)


@pytest.mark.parametrize("seed", [10, 11])
def test_random_dense_bd_and_bb(sb, seed):
    """dense_bd / dense_bb: r in dense tails, value-dependent block creation."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Ad, A = rand_bs(rng, (4, 9, 6), 2, density=0.7)          # (p | x, r)
    # zero some r-slices so the creation rule matters
    A_arr = Ad.copy()
    A_arr[:, :, 2] = 0.0
    A_arr[1, :, :] = 0.0
    A_arr[2, :, 1:] = 0.0
    A = so.blocksparse_from_dense(A_arr, 2)
    B = rng.standard_normal((6, 13))                          # (r, y)
    B[1, :] = 0.0
    B[3:, :] = 0.0
    Cg, Cref = run_both(sb, so.BS.empty((4, 9, 13), 2), ["p", "x", "y"], A, ["p", "x", "r"], B, ["r", "y"])
    assert_bs_equal(Cg, Cref)
    Bbs_arr = rng.standard_normal((5, 6, 11))                 # (q | r, z)
    Bbs_arr[0, 0, :] = 0.0
    Bbs_arr[2, :, :] = 0.0
    Bbs = so.blocksparse_from_dense(Bbs_arr, 2)
    A2 = so.blocksparse_from_dense(A_arr, 2)
    Cg, Cref = run_both(sb, so.BS.empty((4, 5, 9, 11), 2), ["p", "q", "x", "z"], A2, ["p", "x", "r"], Bbs,
                        ["q", "r", "z"])
    assert_bs_equal(Cg, Cref)


@pytest.mark.parametrize("seed", [12, 13])
def test_random_coo_paths_bit_exact(sb, seed):
    """COO×Dense, COO×BS (prefix and dense-index) and COO×COO."""
    rng = np.random.Generator(np.random.PCG64(seed))
    _, A = rand_coo(rng, (6, 5, 7))                            # (i, p, r)
    B = rng.standard_normal((9, 7))                            # (x, r)
    Cg, Cref = run_both(sb, so.BS.empty((5, 6, 9), 1), ["p", "i", "x"], A, ["i", "p", "r"], B, ["x", "r"])
    assert_bs_equal(Cg, Cref, exact=True)
    _, Bbs = rand_bs(rng, (7, 3, 4, 5), 2)                     # (r, j | y, z)
    Cg, Cref = run_both(sb, so.BS.empty((6, 5, 3, 4, 5), 2), ["i", "p", "j", "y", "z"], A, ["i", "p", "r"], Bbs,
                        ["r", "j", "y", "z"])
    assert_bs_equal(Cg, Cref, exact=True)
    Bd_arr = rng.standard_normal((3, 4, 7))                    # (j | y, r)
    Bd_arr[:, :, 1] = 0.0
    Bd = so.blocksparse_from_dense(Bd_arr, 2)
    Cg, Cref = run_both(sb, so.BS.empty((6, 5, 3, 4), 1), ["i", "p", "j", "y"], A, ["i", "p", "r"], Bd,
                        ["j", "y", "r"])
    assert_bs_equal(Cg, Cref, exact=True)
    _, Bc = rand_coo(rng, (7, 4))
    Cg, Cref = run_both(sb, so.COO((6, 5, 4)), ["i", "p", "j"], A, ["i", "p", "r"], Bc, ["r", "j"])
    assert Cg.keys == Cref.keys and Cg.vals == Cref.vals


@pytest.mark.parametrize("seed", [14])
def test_random_aliased(sb, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    # COO × Dense → Aliased with demotion
    _, A = rand_coo(rng, (6, 5), density=0.5)
    B = rng.standard_normal((8, 5))
    Cg, Cref = run_both(sb, so.Aliased.empty((6, 8), 1), ["i", "x"], A, ["i", "r"], B, ["x", "r"])
    assert_aliased_equal(Cg, Cref)
    # Aliased × Dense (prefix and dense), Aliased × Aliased (prefix, dense, shared)
    Aarr = rng.standard_normal((4, 3, 6))
    Aarr[1] = Aarr[0] * 1.0
    Aal = so.aliased_from_blocksparse_unique(so.blocksparse_from_dense(Aarr, 1))   # (i, r | x)
    Bd = rng.standard_normal((3, 7))
    Cg, Cref = run_both(sb, so.Aliased.empty((4, 6, 7), 2), ["i", "x", "y"], Aal, ["i", "r", "x"], Bd, ["r", "y"])
    assert_aliased_equal(Cg, Cref)
    Aal2 = so.aliased_from_blocksparse_unique(so.blocksparse_from_dense(rng.standard_normal((4, 6, 3)), 2))
    Cg, Cref = run_both(sb, so.Aliased.empty((4, 6, 7), 2), ["i", "x", "y"], Aal2, ["i", "x", "r"], Bd, ["r", "y"])
    assert_aliased_equal(Cg, Cref)
    Bal = so.aliased_from_blocksparse_unique(so.blocksparse_from_dense(rng.standard_normal((5, 3, 2)), 1))
    Cg, Cref = run_both(sb, so.Aliased.empty((4, 5, 6, 2), 2), ["i", "j", "x", "z"], Aal, ["i", "r", "x"], Bal,
                        ["j", "r", "z"])
    assert_aliased_equal(Cg, Cref)
    Bal2 = so.aliased_from_blocksparse_unique(so.blocksparse_from_dense(rng.standard_normal((5, 2, 3)), 2))
    Cg, Cref = run_both(sb, so.Aliased.empty((4, 5, 6, 2), 2), ["i", "j", "x", "z"], Aal2, ["i", "x", "r"], Bal2,
                        ["j", "z", "r"])
    assert_aliased_equal(Cg, Cref)


def test_aliased_shared_paths(sb):
    rng = np.random.Generator(np.random.PCG64(21))
    for case in kc.bs_bs_multi_cases()[:3] + kc.bs_dense_cases()[:2]:
        A = so.aliased_from_blocksparse_unique(so.blocksparse_from_dense(case.A, case.n2A))
        B = case.B if case.kind_B == "dense" else so.aliased_from_blocksparse_unique(
            so.blocksparse_from_dense(case.B, case.n2B))
        Cg, Cref = run_both(sb, so.Aliased.empty(case.dimsC, case.n2C), case.labelsC, A, case.labelsA, B,
                            case.labelsB)
        assert_aliased_equal(Cg, Cref)
    # multi-label aliased × dense with a shared prefix
    Aarr = rng.standard_normal((3, 4, 5, 6))   # (i, q | m, k)
    A = so.aliased_from_blocksparse_unique(so.blocksparse_from_dense(Aarr, 2))
    B = rng.standard_normal((4, 6, 7))          # (q, k, n)
    Cg, Cref = run_both(sb, so.Aliased.empty((3, 5, 7), 2), ["i", "m", "n"], A, ["i", "q", "m", "k"], B,
                        ["q", "k", "n"])
    assert_aliased_equal(Cg, Cref)


def test_bs_bs_to_dense_sink(sb):
    rng = np.random.Generator(np.random.PCG64(31))
    _, A = rand_bs(rng, (3, 4, 5), 1, density=0.8)   # (q, i | k)
    _, B = rand_bs(rng, (3, 5, 6), 2, density=0.8)   # (q | k, n)
    # P_C = 0 output of the reference requires C dense = all of A/B kept dense labels
    Aa = so.blocksparse_from_dense(so.bs_to_dense(A), 2)   # (q | i, k)
    ref = so.contract_bs_bs_to_dense((4, 6), ["i", "n"], Aa, ["q", "i", "k"], B, ["q", "k", "n"])
    got = sb.contract_bs_bs_to_dense((4, 6), ["i", "n"], lib_operand(sb, Aa), ["q", "i", "k"], lib_operand(sb, B),
                                     ["q", "k", "n"]).to_numpy()
    assert rel_err(got, ref) <= RTOL


# ── storage operations on the device ─────────────────────────────────────


def test_conversions_and_permutes(sb):
    rng = np.random.Generator(np.random.PCG64(41))
    D = rng.standard_normal((4, 3, 2, 5)) * (rng.random((4, 3, 1, 1)) < 0.6)
    A = sb.blocksparse_from_dense(D, 2)
    R = so.blocksparse_from_dense(D, 2)
    assert A.keys == R.keys and np.array_equal(A.data, R.data)
    assert np.array_equal(sb.to_dense(A), D)
    for perm in ([2, 1, 3, 4], [1, 2, 4, 3], [2, 1, 4, 3]):
        Ap, Rp = sb.permutedims(A, perm), so.bs_permutedims(R, perm)
        assert Ap.keys == Rp.keys and np.array_equal(Ap.data, Rp.data)
    with pytest.raises(sb.SparseBackendsError):
        sb.permutedims(A, [3, 2, 1, 4])
    Dg = rng.standard_normal((40, 33, 17))
    assert np.array_equal(sb.to_dense(sb.permutedims(sb.DenseTensor(Dg), [3, 1, 2])), np.transpose(Dg, (2, 0, 1)))
    C = sb.coo_from_dense(D, atol=0.0)
    Cr = so.coo_from_dense(D, atol=0.0)
    assert C.keys == Cr.keys and C.vals == Cr.vals
    Cp = sb.sort_(sb.permutedims(C, [3, 1, 2, 4]))
    Crp = so.coo_sort(so.coo_permutedims(Cr, [3, 1, 2, 4]))
    assert Cp.keys == Crp.keys and Cp.vals == Crp.vals
    # rtol thresholding of blocksparse_from_dense
    A2 = sb.blocksparse_from_dense(D, 2, rtol=0.3)
    R2 = so.blocksparse_from_dense(D, 2, rtol=0.3)
    assert A2.keys == R2.keys


def test_error_statuses(sb):
    A = sb.NewBlockSparseSorted.empty((3, 4), 1)
    B = sb.DenseTensor(np.zeros((5, 2)))
    C = sb.NewBlockSparseSorted.empty((3, 2), 1)
    with pytest.raises(sb.SparseBackendsError) as ei:
        sb.contract_(C, ["i", "y"], A, ["i", "r"], B, ["r", "y"])   # dims 4 vs 5
    assert ei.value.status == "SB_ERR_DIM_MISMATCH"
    Cc = sb.COOTensor((3, 2))
    with pytest.raises(sb.SparseBackendsError) as ei:
        sb.contract_(Cc, ["i", "y"], A, ["i", "r"], sb.DenseTensor(np.zeros((4, 2))), ["r", "y"])
    assert ei.value.status == "SB_ERR_UNSUPPORTED_TYPES"


def test_context_destroy_is_deferred_while_tensors_live(sb):
    """sb_ctx_destroy with live tensors is deferred to the last sb_tensor_free
    (Python finalizers can run in any order, e.g. at interpreter exit)."""
    import ctypes as C
    ctx = sb.Context(0)
    lib = ctx._lib
    t = sb.NewBlockSparseSorted((2, 3), 1, [(1,)], None, np.arange(3.0), ctx=ctx)
    u = sb.DenseTensor(np.ones((2, 2)), ctx)
    h = ctx._h
    assert lib.sb_ctx_destroy(h) == 0           # deferred: two tensors alive
    assert np.array_equal(t.data, np.arange(3.0))  # the context still works for them
    del u
    ctx._h = C.c_void_p()                       # Python must not destroy it again
    del t                                       # the last free destroys the context


@pytest.mark.parametrize("seed", [51, 52])
def test_random_skinny_streaming_gemm(sb, seed):
    """Small K and one small output side route to the streaming GEMM kernel
    (both orientations, several pairs accumulated per output block)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    # A[(i, q) | (m, k)] x B[(q, j) | (k, n)]: M=700 rows, K=13, N=11
    _, A = rand_bs(rng, (2, 3, 700, 13), 2, density=0.9)
    _, B = rand_bs(rng, (3, 2, 13, 11), 2, density=0.9)
    lA, lB = ["i", "q", "m", "k"], ["q", "j", "k", "n"]
    for lC, dims in ((["i", "j", "m", "n"], (2, 2, 700, 11)), (["i", "j", "n", "m"], (2, 2, 11, 700))):
        Cg, Cref = run_both(sb, so.BS.empty(dims, 2), lC, A, lA, B, lB)
        assert_bs_equal(Cg, Cref)


@pytest.mark.parametrize("seed", [61, 62])
def test_random_splitk_gemm(sb, seed):
    """Few output tiles with long reductions take the split-K path (partial
    tiles summed in a fixed order by a second kernel)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    _, A = rand_bs(rng, (2, 3, 70, 1100), 2, density=1.0)
    _, B = rand_bs(rng, (3, 2, 1100, 50), 2, density=1.0)
    lA, lB = ["i", "q", "m", "k"], ["q", "j", "k", "n"]
    for lC, dims in ((["i", "j", "m", "n"], (2, 2, 70, 50)), (["i", "j", "n", "m"], (2, 2, 50, 70))):
        Cg, Cref = run_both(sb, so.BS.empty(dims, 2), lC, A, lA, B, lB)
        assert_bs_equal(Cg, Cref)


def test_is_dense_matches_oracle():
    import sparsebackends_b200 as sb
    rng = np.random.Generator(np.random.PCG64(8))
    for density in (1.0, 0.5):
        A = rng.standard_normal((3, 2, 4, 5)) * (rng.random((3, 2, 1, 1)) < density)
        Bo = so.blocksparse_from_dense(A, 2)
        Bg = sb.NewBlockSparseSorted(Bo.dims, 2, Bo.keys, Bo.ids, Bo.data)
        assert sb.is_dense(Bg) == so.bs_is_dense(Bo)
    assert sb.is_dense(sb.DenseTensor(np.ones((2, 3))))
