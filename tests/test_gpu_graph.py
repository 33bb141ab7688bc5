"""CUDA graph capture of library calls (sb_ctx_capture_begin/end, sb_graph_launch).

* a captured H_eff chain replays to the same bits as the eager chain, for the
  ragged and the uniform layout, and follows new input values written into the
  captured input tensor;
* the Lanczos eigensolver on a graph-replayed operator gives the same Ritz
  value and vector as on the eager operator;
* a call that reads values back to the host (value-dependent block creation)
  cannot be captured: the capture fails with an error status and the context
  keeps working for eager calls;
* a capture that holds the first kernel launches of a process (kernel
  attributes and persistent grid sizes are set up then) replays to the eager
  result.
"""
import numpy as np
import pytest

from tests.heff_dense import small_layout

pytestmark = pytest.mark.gpu


def _setup(ragged, seed=41, chi=24):
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    lay = small_layout(chi)
    rng = np.random.Generator(np.random.PCG64(seed))
    ops = qn.hermitian_operators(lay, rng)
    pk, pd, pe = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    ctx = sb.Context(0)

    def dev(name, k, d, e):
        if ragged:
            return sb.NewBlockSparseSorted(lay.dims[name], lay.n2[name], k, None, d, ctx=ctx, block_dims=e)
        return sb.NewBlockSparseSorted(lay.dims[name], lay.n2[name], k, None, qn.pad_ragged(lay, name, k, d, e),
                                       ctx=ctx)

    T = {n: dev(n, *v) for n, v in ops.items()}
    psi = dev("psi", pk, pd, pe)
    return sb, qn, lay, ctx, T, psi, rng


@pytest.mark.parametrize("ragged", [True, False])
def test_graph_replay_matches_eager(ragged):
    sb, qn, lay, ctx, T, psi, rng = _setup(ragged)
    eager = qn.HeffChain(lay, ctx)
    want = eager.apply(psi, T["L"], T["W1"], T["W2"], T["R"]).data
    chain = qn.HeffChain(lay, ctx)
    g = chain.capture(psi, T["L"], T["W1"], T["W2"], T["R"])
    sb.fill_(chain.out["T4"], 0.0)
    g.launch()
    assert np.array_equal(chain.out["T4"].data, want)
    # new input values through the captured input tensor
    x2 = sb.copy(psi)
    sb.scale_(x2, -0.5)
    sb.axpy_(1.0, sb.similar(psi), x2)
    sb.map_(psi, x2, sb.MAP_COPY)
    g.launch()
    want2 = eager.apply(psi, T["L"], T["W1"], T["W2"], T["R"]).data
    assert np.array_equal(chain.out["T4"].data, want2)
    for _ in range(3):
        g.launch()
    assert np.array_equal(chain.out["T4"].data, want2)


def test_lanczos_on_graph_operator():
    sb, qn, lay, ctx, T, psi, rng = _setup(True, seed=42)
    from sparsebackends_b200 import krylov
    op = qn.HeffOperator(lay, T["L"], T["W1"], T["W2"], T["R"], ctx)
    opg = qn.HeffOperator(lay, T["L"], T["W1"], T["W2"], T["R"], ctx, graph_like=psi)
    v1, x1, _ = krylov.eigsolve(op, psi, 1, "SR", krylovdim=6, maxiter=2, tol=1e-14)
    v2, x2, _ = krylov.eigsolve(opg, psi, 1, "SR", krylovdim=6, maxiter=2, tol=1e-14)
    assert v1[0] == v2[0]
    assert np.array_equal(x1[0].data, x2[0].data)


def test_capture_of_a_readback_call_fails_cleanly():
    import sparsebackends_b200 as sb
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(5))
    A = sb.blocksparse_from_dense(rng.standard_normal((3, 4, 5)), 2, ctx=ctx)   # (p | x, r)
    B = sb.blocksparse_from_dense(rng.standard_normal((2, 5, 6)), 2, ctx=ctx)   # (q | r, y)
    C = sb.NewBlockSparseSorted.empty((3, 2, 4, 6), 2, ctx=ctx)
    lab = (["p", "q", "x", "y"], ["p", "x", "r"], ["q", "r", "y"])
    sb.contract_(C, lab[0], A, lab[1], B, lab[2])  # dense_bb: value-dependent block creation
    want = C.data
    with pytest.raises(sb.SparseBackendsError):
        ctx.capture(lambda: sb.contract_(C, lab[0], A, lab[1], B, lab[2]))
    C2 = sb.NewBlockSparseSorted.empty((3, 2, 4, 6), 2, ctx=ctx)
    sb.contract_(C2, lab[0], A, lab[1], B, lab[2])
    assert np.array_equal(C2.data, want)


_FIRST_CALL_CAPTURED = r"""
import sys
sys.path.insert(0, {root!r})
import numpy as np
from tests.test_gpu_graph import _setup
sb, qn, lay, ctx, T, psi, rng = _setup({ragged}, chi=64)
chain = qn.HeffChain(lay, ctx)
# no eager call before: the GEMM kernels' first launches of this process are captured
g = ctx.capture(lambda: chain.apply(psi, T["L"], T["W1"], T["W2"], T["R"]),
                keep=[psi, T["L"], T["W1"], T["W2"], T["R"], *chain.out.values()])
g.launch()
got = chain.out["T4"].data
eager = qn.HeffChain(lay, ctx)
want = eager.apply(psi, T["L"], T["W1"], T["W2"], T["R"]).data
assert np.array_equal(got, want)
del g
print("ok")
"""


@pytest.mark.parametrize("ragged", [True, False])
def test_capture_as_the_first_launches_of_a_process(ragged):
    """Kernel attributes and persistent-grid sizes are set up on a kernel's
    first launch; a capture that holds those first launches (a fresh process,
    nothing run eagerly before) must replay to the eager result."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", _FIRST_CALL_CAPTURED.format(root=root, ragged=ragged)],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and out.stdout.strip().endswith("ok"), out.stderr[-2000:]
