"""The C++ restatement of contract_shared! (``oracle/cpu_ref``, the CPU
baseline of the benchmark) against the numpy oracle: the H_eff chain and
environment contractions of the N = 16 centre problem and of the J1-J2-sized
problem (``tests/join_cases.py``), the PXP chain's two dense contractions, and
the error paths the reference asserts."""
import numpy as np
import pytest

from oracle import cpu_ref
from oracle import sparse_oracle as so
from tests import join_cases as jc


@pytest.fixture(scope="module", autouse=True)
def built():
    cpu_ref.build()
    cpu_ref.load()


def _cases():
    return jc.centre_problem_cases() + jc.j1j2_sized_cases()


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_matches_numpy_oracle(case):
    name, C0, lc, A, la, B, lb = case
    ref = so.contract(so.BS.empty(C0.dims, C0.n2), lc, A, la, B, lb)
    got = cpu_ref.contract_shared(C0, lc, A, la, B, lb)
    assert got.keys == ref.keys, name
    rb, gb = ref.blocks_by_key(), got.blocks_by_key()
    scale = max((np.max(np.abs(v)) for v in rb.values()), default=1.0)
    for k, v in rb.items():
        assert np.max(np.abs(gb[k] - v)) <= 1e-13 * scale, (name, k)


def test_pxp_dense_steps():
    """The two contract_shared! steps of the PXP matvec (L*psi and T3*R)."""
    from oracle.pxp_oracle import OracleProblem, o_run
    from sparsebackends_b200 import pxp
    prob = OracleProblem(12, 16, 5)
    t = o_run(pxp.HEFF_STEPS, {"psi": prob.psi, "L": prob.L, "R": prob.R, "W1f": prob.Wf, "W2f": prob.Wf})
    lab = dict(pxp.LABELS)
    lab.update({"T3": pxp.HEFF_STEPS[4][2]})
    for c, a, b, lc in (("T1", "L", "psi", pxp.HEFF_STEPS[0][2]), ("T4", "T3", "R", pxp.HEFF_STEPS[5][2])):
        ops = {"L": prob.L, "psi": prob.psi, "R": prob.R, "T3": t["T3"]}
        got = cpu_ref.contract_shared(t[c], list(lc), ops[a], list(lab[a]), ops[b], list(lab[b]))
        assert got.keys == t[c].keys
        for k, v in t[c].blocks_by_key().items():
            assert np.max(np.abs(got.blocks_by_key()[k] - v)) <= 1e-13 * max(1.0, np.max(np.abs(v)))


def test_rejects_interleaved_dense_tail():
    rng = np.random.Generator(np.random.PCG64(3))
    A = so.blocksparse_from_dense(rng.standard_normal((2, 3, 4, 5)), 2)   # (p, q | m, k)
    B = so.blocksparse_from_dense(rng.standard_normal((3, 2, 5, 6)), 2)   # (q, r | k, n)
    C0 = so.BS.empty((2, 2, 4, 6), 2)
    # C tail [m, n, t] interleaves A's kept labels (m, t) with B's (n)
    A3 = so.blocksparse_from_dense(rng.standard_normal((2, 3, 4, 5, 2)), 3)  # (p, q | m, k, t)
    with pytest.raises(RuntimeError, match="interleaves"):
        cpu_ref.contract_shared(so.BS.empty((2, 2, 4, 6, 2), 3), ["p", "r", "m", "n", "t"], A3,
                                ["p", "q", "m", "k", "t"], B, ["q", "r", "k", "n"])
    # C tail [n, m] (B's kept label, then A's) is allowed
    got = cpu_ref.contract_shared(C0, ["p", "r", "n", "m"], A, ["p", "q", "m", "k"], B, ["q", "r", "k", "n"])
    ref = so.contract(so.BS.empty((2, 2, 6, 4), 2), ["p", "r", "n", "m"], A, ["p", "q", "m", "k"], B,
                      ["q", "r", "k", "n"])
    assert got.keys == ref.keys


def test_rejects_shared_label_across_prefix_and_tail():
    rng = np.random.Generator(np.random.PCG64(4))
    A = so.blocksparse_from_dense(rng.standard_normal((2, 3, 4)), 1)   # (p, q | m)
    B = so.blocksparse_from_dense(rng.standard_normal((3, 2, 4)), 2)   # (q | p, m)
    with pytest.raises(RuntimeError, match="crosses"):
        cpu_ref.contract_shared(so.BS.empty((1,), 1), ["z"], A, ["p", "q", "m"], B, ["q", "p", "m"])


def test_heff_chain_matches_numpy_oracle():
    """The four-step H_eff chain of the benchmark (uniform reference layout,
    small chi) through the C++ restatement, as bench.py's CPU baseline runs it."""
    import bench
    from sparsebackends_b200 import qn
    layout = bench.workload(48)
    host = bench.host_tensors(layout, 7)
    keep_np, keep_cpp = [], []
    bench.cpu_matvec_rate(layout, host, 0.0, 1, keep=keep_np)
    bench.cpp_matvec_rate(layout, host, 0.0, 1, keep=keep_cpp)
    ref, got = keep_np[0], keep_cpp[0].to_bs()
    assert got.keys == ref.keys
    rb, gb = ref.blocks_by_key(), got.blocks_by_key()
    scale = max(np.max(np.abs(v)) for v in rb.values())
    assert max(np.max(np.abs(gb[k] - v)) for k, v in rb.items()) <= 1e-12 * scale


def test_pxp_matvec_matches_numpy_oracle():
    """The whole PXP matvec (contract_shared!, fuse_two_axes!, contract_prefix!)
    through the C++ restatement, as the PXP leg's CPU baseline runs it."""
    from oracle.pxp_oracle import OracleProblem, o_run
    from sparsebackends_b200 import pxp
    prob = OracleProblem(12, 16, 5)
    apply, psi = cpu_ref.pxp_heff_runner(prob)
    got = apply(psi).to_bs()
    ref = prob.apply(prob.psi)
    assert got.keys == ref.keys
    for k, v in ref.blocks_by_key().items():
        assert np.max(np.abs(got.blocks_by_key()[k] - v)) <= 1e-13 * max(1.0, np.max(np.abs(v))), k
    # the scaled adds alone are bit-exact: T2 from the oracle's own T1f
    t = o_run(pxp.HEFF_STEPS, {"psi": prob.psi, "L": prob.L, "R": prob.R, "W1f": prob.Wf, "W2f": prob.Wf})
    t1f = cpu_ref.Tensor.from_bs(t["T1f"])
    t2 = cpu_ref.contract_coo_prefix(t["T2"].dims, 2, list(pxp.HEFF_STEPS[2][2]), prob.Wf,
                                     list(pxp.LABELS["W1f"]), t1f, ["qlp", "s2", "qr", "x1", "lp", "r"]).to_bs()
    assert t2.keys == t["T2"].keys
    for k, v in t["T2"].blocks_by_key().items():
        assert np.array_equal(t2.blocks_by_key()[k], v), k


def test_fuse_prefix_matches_oracle():
    rng = np.random.Generator(np.random.PCG64(8))
    A = so.blocksparse_from_dense(rng.standard_normal((2, 3, 4, 5, 6)) * (rng.random((2, 3, 4, 1, 1)) < 0.6), 2)
    for ax1, ax2 in ((1, 2), (2, 3), (2, 1)):
        got = cpu_ref.fuse_prefix(cpu_ref.Tensor.from_bs(A), ax1, ax2).to_bs()
        ref = so.fuse_two_axes(A, ax1, ax2)
        assert got.dims == ref.dims
        rb = ref.blocks_by_key()
        assert sorted(got.keys, key=lambda k: k[::-1]) == got.keys and set(got.keys) == set(rb)
        for k, v in rb.items():
            assert np.array_equal(got.blocks_by_key()[k], v)
