"""Tensor-core (tcgen05) block GEMMs of sb_contract against the CPU oracle.

The reference multiplies every matched block pair with an FP64 ``mul!``
(``contract_bs_bs.jl:716-723``, ``contract_bs_dense.jl:576-611``).  With a
context in SB_PRECISION_TF32X3 the same contractions run on the tcgen05
tensor cores with every FP64 operand split into TF32 hi + lo parts and FP32
accumulation; SB_PRECISION_TF32 multiplies once in TF32.  Block structure
must stay bit-identical to the oracle's; values are held to a per-block
relative Frobenius error of TOL_X3 (3xTF32) and TOL_1 (TF32).

Shapes cover both tile orientations (the long side of C on the 128-row side
or on the <= 256-row side), several 128-row and 256-row tiles per block,
k extents that are not multiples of the 32-deep k-tile, several pairs per
output block (the pair K loops are concatenated), and both operand
orders (transposed and untransposed global layouts).
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so

pytestmark = pytest.mark.gpu

TOL_X3 = 2e-5   # 3xTF32: ~22 significant bits per operand, FP32 accumulation over K terms
TOL_1 = 4e-3    # single TF32 product: 11 significant bits


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as sbmod
    return sbmod


@pytest.fixture(scope="module")
def ctxs(sb):
    out = {}
    for p in ("f64", "tf32x3", "tf32"):
        c = sb.Context(0)
        c.set_precision(p)
        out[p] = c
    return out


def rel_err(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def rand_bs(rng, dims, n2, density=0.8):
    P = len(dims) - n2
    A = rng.standard_normal(dims)
    mask = rng.random(dims[:P]) < density
    A = A * mask.reshape(dims[:P] + (1,) * n2)
    return so.blocksparse_from_dense(A, n2)


def run(sb, ctx, C0, lC, A, lA, B, lB):
    Cg = sb.NewBlockSparseSorted.empty(C0.dims, C0.n2, ctx=ctx)
    sb.contract_(Cg, lC, sb.NewBlockSparseSorted(A.dims, A.n2, A.keys, A.ids, A.data, ctx=ctx), lA,
                 sb.NewBlockSparseSorted(B.dims, B.n2, B.keys, B.ids, B.data, ctx=ctx), lB)
    ctx.synchronize()  # raises SB_ERR_TIMEOUT if a bounded tensor-core wait ran out
    return Cg


def check(Cg, Cref, tol):
    assert Cg.keys == Cref.keys and len(Cref.keys) > 0
    gb, rb = Cg.blocks_by_key(), Cref.blocks_by_key()
    worst = 0.0
    for k, v in rb.items():
        e = rel_err(gb[k], v)
        worst = max(worst, e)
        assert e <= tol, (k, e)
    return worst


# (I, Q, J, M, K, N): C[(i, j) | (m, n)] = sum_q A[(i, q) | (m, k)] B[(q, j) | (k, n)]
SHAPES = [
    (2, 3, 2, 300, 77, 40),    # long M, short N
    (2, 3, 2, 40, 77, 300),    # short M, long N
    (1, 2, 2, 263, 45, 270),   # several tiles on both sides
    (3, 2, 1, 129, 31, 17),    # one row past a 128-row tile, K below one k-tile
    (2, 4, 2, 64, 200, 64),    # long concatenated K (split into k-segments)
    (1, 3, 1, 200, 1500, 150), # several FP32 chunks per segment (Kahan-summed) and several segments
    (3, 1, 3, 1024, 48, 1200), # over four tiles per SM: no k-segments
]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("order", ["ijmn", "jinm"])
@pytest.mark.parametrize("prec", ["tf32x3", "tf32"])
def test_tc_shared_bb_matches_oracle(sb, ctxs, shape, order, prec):
    I, Q, J, M, K, N = shape
    rng = np.random.Generator(np.random.PCG64(sum(shape) * 7 + (order == "ijmn")))
    A = rand_bs(rng, (I, Q, M, K), 2)
    B = rand_bs(rng, (Q, J, K, N), 2)
    lC = ["i", "j", "m", "n"] if order == "ijmn" else ["j", "i", "n", "m"]
    ext = {"i": I, "j": J, "m": M, "n": N}
    C0 = so.BS.empty(tuple(ext[l] for l in lC), 2)
    lA, lB = ["i", "q", "m", "k"], ["q", "j", "k", "n"]
    Cref = so.contract(C0, lC, A, lA, B, lB)
    Cg = run(sb, ctxs[prec], C0, lC, A, lA, B, lB)
    worst = check(Cg, Cref, TOL_X3 if prec == "tf32x3" else TOL_1)
    # the FP64 path on the same context family stays at the drop-in tolerance
    Cf = run(sb, ctxs["f64"], C0, lC, A, lA, B, lB)
    check(Cf, Cref, 1e-12)
    print(f"{prec} {shape} {order}: worst block rel err {worst:.2e}")


def test_tc_bit_reproducible(sb, ctxs):
    """Fixed tile order and accumulation order: repeated calls give identical bits."""
    rng = np.random.Generator(np.random.PCG64(11))
    A = rand_bs(rng, (2, 3, 150, 90), 2)
    B = rand_bs(rng, (3, 2, 90, 70), 2)
    lC, lA, lB = ["i", "j", "m", "n"], ["i", "q", "m", "k"], ["q", "j", "k", "n"]
    C0 = so.BS.empty((2, 2, 150, 70), 2)
    a = run(sb, ctxs["tf32x3"], C0, lC, A, lA, B, lB).blocks_by_key()
    b = run(sb, ctxs["tf32x3"], C0, lC, A, lA, B, lB).blocks_by_key()
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_tc_shared_bd_matches_oracle(sb, ctxs):
    """BS x Dense contract_shared! (contract_bs_dense.jl:411-619) on the tensor cores."""
    rng = np.random.Generator(np.random.PCG64(21))
    d, w, X, Y = 2, 9, 140, 70
    W = rand_bs(rng, (d, d, w, w), 2, density=0.8)
    T = rng.standard_normal((d, w, X, Y))
    lC = ["sp", "wr", "x", "y"]
    C0 = so.BS.empty((d, w, X, Y), 3)
    Cref = so.contract(C0, lC, W, ["sp", "s", "wl", "wr"], T, ["s", "wl", "x", "y"])
    ctx = ctxs["tf32x3"]
    Cg = sb.NewBlockSparseSorted.empty(C0.dims, C0.n2, ctx=ctx)
    sb.contract_(Cg, lC, sb.NewBlockSparseSorted(W.dims, W.n2, W.keys, W.ids, W.data, ctx=ctx),
                 ["sp", "s", "wl", "wr"], sb.DenseTensor(T, ctx=ctx), ["s", "wl", "x", "y"])
    ctx.synchronize()
    check(Cg, Cref, TOL_X3)


def _layout_small():
    from sparsebackends_b200 import qn
    left = qn.U1Link([-5, -3, -1, 1, 3, 5], [2, 8, 22, 22, 8, 2])
    right = qn.U1Link([-3, -1, 1, 3], [7, 25, 25, 7])
    mpo = qn.mpo_link({-2: 1, 0: 3, 2: 1})
    return qn.HeffLayout(left, right, mpo)


@pytest.mark.parametrize("ragged,f32,w12", [(True, False, False), (False, False, False), (True, True, False),
                                            (True, True, True)])
def test_tc_heff_chain_matches_oracle(sb, ctxs, ragged, f32, w12):
    """The two-site H_eff chain (psi*L, *W1, *W2, *R) with its tiled steps on
    the tensor cores, against the oracle's FP64 chain on the padded tensors;
    also with FP32-stored intermediates (T1, T2, T3) and in the W12 order."""
    from sparsebackends_b200 import qn
    lay = _layout_small()
    ctx = ctxs["tf32x3"]
    rng = np.random.Generator(np.random.PCG64(5))
    dev, pad = {}, {}
    for name in ("psi", "L", "W1", "W2", "R"):
        keys, data, exts = qn.random_block_tensor(lay, name, rng, 0.5, ragged=True)
        padded = qn.pad_ragged(lay, name, keys, data, exts)
        pad[name] = (keys, padded)
        if ragged:
            dev[name] = sb.NewBlockSparseSorted(lay.dims[name], lay.n2[name], keys, None, data, ctx=ctx,
                                                block_dims=exts)
        else:
            dev[name] = sb.NewBlockSparseSorted(lay.dims[name], lay.n2[name], keys, None, padded, ctx=ctx)
    chain = qn.HeffChain(lay, ctx=ctx, w12=w12, f32_intermediates=f32)
    out = chain.apply(dev["psi"], dev["L"], dev["W1"], dev["W2"], dev["R"])
    ctx.synchronize()
    assert chain.out["T1"].is_f32 == f32 and not out.is_f32
    got = sb.to_uniform(out) if ragged else out
    t = {n: so.BS(lay.dims[n], lay.n2[n], k, list(range(1, len(k) + 1)), d) for n, (k, d) in pad.items()}
    lab = lay.labels
    for c, a, b in qn.HeffChain.STEPS:
        t[c] = so.contract(so.BS.empty(lay.dims[c], lay.n2[c]), lab[c], t[a], lab[a], t[b], lab[b])
    check(got, t["T4"], TOL_X3)


def test_tc_precision_api(sb):
    c = sb.Context(0)
    assert c.precision == "f64"
    c.set_precision("tf32x3")
    assert c.precision == "tf32x3"
    with pytest.raises(KeyError):
        c.set_precision("fp8")
    st = c._lib.sb_ctx_set_precision(c._h, 7)
    assert st == 1  # SB_ERR_INVALID_ARG
    c.set_precision("f64")
    assert c.precision == "f64"


def test_f32_tensors_rejected_outside_the_chain_kernels(sb, ctxs):
    """FP32 storage is accepted only by contract_shared! BS x BS launches that
    can read or write it; elsewhere the library reports SB_ERR_UNSUPPORTED_TYPES."""
    ctx = ctxs["f64"]
    rng = np.random.Generator(np.random.PCG64(3))
    A = rand_bs(rng, (2, 3, 20, 30), 2)
    B = rand_bs(rng, (3, 2, 30, 10), 2)
    C = sb.NewBlockSparseSorted.empty((2, 2, 20, 10), 2, ctx=ctx, f32=True)
    assert C.is_f32
    with pytest.raises(sb.SparseBackendsError) as ei:
        sb.contract_(C, ["i", "j", "m", "n"], sb.NewBlockSparseSorted(A.dims, 2, A.keys, A.ids, A.data, ctx=ctx),
                     ["i", "q", "m", "k"], sb.NewBlockSparseSorted(B.dims, 2, B.keys, B.ids, B.data, ctx=ctx),
                     ["q", "j", "k", "n"])
    assert ei.value.status == "SB_ERR_UNSUPPORTED_TYPES"
    # the same call on a tensor-core context writes FP32 values
    c2 = ctxs["tf32x3"]
    C2 = sb.NewBlockSparseSorted.empty((2, 2, 20, 10), 2, ctx=c2, f32=True)
    sb.contract_(C2, ["i", "j", "m", "n"], sb.NewBlockSparseSorted(A.dims, 2, A.keys, A.ids, A.data, ctx=c2),
                 ["i", "q", "m", "k"], sb.NewBlockSparseSorted(B.dims, 2, B.keys, B.ids, B.data, ctx=c2),
                 ["q", "j", "k", "n"])
    Cref = so.contract(so.BS.empty((2, 2, 20, 10), 2), ["i", "j", "m", "n"], A, ["i", "q", "m", "k"], B,
                       ["q", "j", "k", "n"])
    check(C2, Cref, TOL_X3)


def _pair(sb, ctx, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    A = rand_bs(rng, (2, 3, 150, 90), 2)
    B = rand_bs(rng, (3, 2, 90, 70), 2)
    a = sb.NewBlockSparseSorted(A.dims, 2, A.keys, A.ids, A.data, ctx=ctx)
    b = sb.NewBlockSparseSorted(B.dims, 2, B.keys, B.ids, B.data, ctx=ctx)
    return a, b


LC, LA, LB = ["i", "j", "m", "n"], ["i", "q", "m", "k"], ["q", "j", "k", "n"]


def test_tc_packed_operands_follow_writes(sb, ctxs):
    """The packed (split, swizzled) operand images are reused while an operand
    is unchanged and rebuilt after a library call writes it: scaling A by 2 in
    place doubles C exactly (the split of 2x is the split of x, doubled)."""
    ctx = ctxs["tf32x3"]
    a, b = _pair(sb, ctx, 31)
    C = sb.NewBlockSparseSorted.empty((2, 2, 150, 70), 2, ctx=ctx)
    sb.contract_(C, LC, a, LA, b, LB)
    c1 = np.array(C.data, copy=True)
    sb.contract_(C, LC, a, LA, b, LB)  # unchanged operands: cached images
    assert np.array_equal(np.array(C.data), c1)
    sb.scale_(a, 2.0)
    sb.contract_(C, LC, a, LA, b, LB)
    assert np.array_equal(np.array(C.data), 2.0 * c1)
    sb.fill_(a, 0.0)
    sb.contract_(C, LC, a, LA, b, LB)
    ctx.synchronize()
    assert not np.any(np.array(C.data))


def test_tc_graph_replay_reads_current_values(sb, ctxs):
    """A captured tensor-core contraction packs its operands inside the graph:
    a replay after an in-place write of an operand uses the new values."""
    ctx = ctxs["tf32x3"]
    a, b = _pair(sb, ctx, 33)
    C = sb.NewBlockSparseSorted.empty((2, 2, 150, 70), 2, ctx=ctx)
    sb.contract_(C, LC, a, LA, b, LB)
    c1 = np.array(C.data, copy=True)
    g = ctx.capture(lambda: sb.contract_(C, LC, a, LA, b, LB), keep=(a, b, C))
    g.launch()
    ctx.synchronize()
    assert np.array_equal(np.array(C.data), c1)
    sb.scale_(b, 0.5)
    g.launch()
    ctx.synchronize()
    assert np.array_equal(np.array(C.data), 0.5 * c1)
    del g
