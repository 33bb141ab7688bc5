"""The allocation-free entry point sb_block_gemm_f64_noalloc.

It serves callers that cannot allocate device memory during a solve (a fixed
pool or budget, or a host runtime that owns the device and forbids cudaMalloc):
they hand in device buffers for inputs and outputs, and the plan goes into the
library's static device scratch array instead of allocated buffers.

Checked here through the C ABI
* against the existing entry point sb_contract (same block-sparse
  contraction, contract_shared! semantics) on two calls in a row;
* against the CPU oracle's contraction (numpy products of the oracle's blocks)
  for every tile shape the entry point picks (64x64, 128x32, 32x128, 128x64,
  64x128), all four operand orders (x_trans, y_trans), pairs of different K
  and padded leading dimensions feeding one output block, and an output block
  with no pairs (written as zeros);
within the GEMM tolerance the parity tests use (1e-12 relative Frobenius per
block); plus the size limit and the argument checks.  The file sorts last so
that a run stopping at the first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import sparse_oracle as so

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _case(seed, I, Q, J, M, K, N):
    """A[(i, q) | (m, k)] x B[(j, q) | (k, n)] -> C[(i, j) | (m, n)]: the
    operands are already in join order, so sb_contract runs one GEMM launch."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Ad = rng.standard_normal((I, Q, M, K)) * (rng.random((I, Q, 1, 1)) < 0.7)
    Bd = rng.standard_normal((J, Q, K, N)) * (rng.random((J, Q, 1, 1)) < 0.7)
    return so.blocksparse_from_dense(Ad, 2), so.blocksparse_from_dense(Bd, 2)


def _plan(A, B, dimsC):
    """Block-pair plan in the order sb_contract uses: C blocks sorted by key,
    pairs within a block in merge-join order."""
    pairs = {}
    for ia, ka in enumerate(A.keys):
        for ib, kb in enumerate(B.keys):
            if ka[1] == kb[1]:
                pairs.setdefault((ka[0], kb[0]), []).append((ia, ib))
    ckeys = sorted(pairs, key=lambda k: (k[1] - 1) * dimsC[0] + (k[0] - 1))
    return ckeys, [pairs[k] for k in ckeys]


def _call(lib, stream, dX, dY, dC, c_off, rows, cols, pbegin, xo, yo, Ks, ldx, ldy, xt, yt):
    nc, npairs = len(c_off), len(xo)
    n1 = max(npairs, 1)
    err = C.create_string_buffer(256)
    st = lib.sb_block_gemm_f64_noalloc(
        C.c_void_p(stream), C.c_void_p(dX), C.c_void_p(dY), C.c_void_p(dC), nc, (C.c_int64 * nc)(*c_off),
        (C.c_int32 * nc)(*rows), (C.c_int32 * nc)(*cols), (C.c_int32 * (nc + 1))(*pbegin),
        (C.c_int64 * n1)(*xo), (C.c_int64 * n1)(*yo), (C.c_int32 * n1)(*Ks), (C.c_int32 * n1)(*ldx),
        (C.c_int32 * n1)(*ldy), xt, yt, err, 256)
    return st, err.value.decode()


def test_noalloc_matches_sb_contract_on_two_calls():
    import sparsebackends_b200 as sb
    ctx = sb.Context(0)
    shapes = [(1, 3, 4, 3, 37, 29, 21), (2, 2, 3, 2, 130, 17, 9)]  # (seed, I, Q, J, M, K, N)
    for seed, I, Q, J, M, K, N in shapes:
        A, B = _case(seed, I, Q, J, M, K, N)
        lA, lB, lC = ["i", "q", "m", "k"], ["j", "q", "k", "n"], ["i", "j", "m", "n"]
        A_t = sb.NewBlockSparseSorted(A.dims, 2, A.keys, A.ids, A.data, ctx=ctx)
        B_t = sb.NewBlockSparseSorted(B.dims, 2, B.keys, B.ids, B.data, ctx=ctx)
        C_ref = sb.NewBlockSparseSorted.empty((I, J, M, N), 2, ctx=ctx)
        sb.contract_(C_ref, lC, A_t, lA, B_t, lB)   # the existing entry point
        C_orc = so.contract(so.BS.empty((I, J, M, N), 2), lC, A, lA, B, lB)  # the CPU oracle
        ckeys, plist = _plan(A, B, (I, J))
        assert C_ref.keys == ckeys == C_orc.keys
        out = sb.DenseTensor(ctx=ctx, dims=(max(len(ckeys) * M * N, 1),))
        pb, xo, yo = [0], [], []
        for pl in plist:
            for ia, ib in pl:
                xo.append(ia * M * K)
                yo.append(ib * K * N)
            pb.append(len(xo))
        nc, npr = len(ckeys), len(xo)
        st, msg = _call(ctx._lib, ctx.stream, A_t.device_ptr()[0], B_t.device_ptr()[0], out.device_ptr()[0],
                        [c * M * N for c in range(nc)], [M] * nc, [N] * nc, pb, xo, yo, [K] * npr, [M] * npr,
                        [K] * npr, 0, 0)
        assert st == 0, msg
        ctx.synchronize()
        got, ref, blk = out.to_numpy(), C_ref.data, M * N
        orc = C_orc.blocks_by_key()
        for c in range(nc):
            g, r = got[c * blk:(c + 1) * blk], ref[c * blk:(c + 1) * blk]
            o = np.asarray(orc[ckeys[c]]).reshape(-1, order="F")
            assert np.linalg.norm(g - r) <= RTOL * max(np.linalg.norm(r), 1e-300)
            assert np.linalg.norm(g - o) <= RTOL * max(np.linalg.norm(o), 1e-300)


def _pairs_sum(pairs):
    """C = sum_p X_p @ Y_p in pair order: the oracle's per-pair accumulation of
    contract_shared_bb (``Cm += Amat @ Bmat``), on blocks of different K."""
    c = np.zeros((pairs[0][0].shape[0], pairs[0][1].shape[1]))
    for x, y in pairs:
        c += x @ y
    return c


def _pack(mats, trans, pad):
    """Concatenate matrices column-major (transposed when ``trans``) with the
    leading dimension padded by ``pad``; returns (flat, offsets, lds)."""
    flat, offs, lds = [], [], []
    off = 0
    for m in mats:
        s = m.T if trans else m
        ld = s.shape[0] + pad
        buf = np.zeros((ld, s.shape[1]))
        buf[: s.shape[0]] = s
        flat.append(buf.reshape(-1, order="F"))
        offs.append(off)
        lds.append(ld)
        off += buf.size
    return np.concatenate(flat), offs, lds


@pytest.mark.parametrize("xt,yt", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N", [(37, 21), (130, 9), (20, 140), (300, 150), (150, 300)])
def test_noalloc_against_oracle_products(xt, yt, M, N):
    """C block 0: two pairs of different K (17 and 40) with padded leading
    dimensions; C block 1: one pair; C block 2: no pairs (zeros).  Two calls
    in a row (the second with the operands scaled) reuse the scratch."""
    import sparsebackends_b200 as sb
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(M * 7 + N + 2 * xt + yt))
    Ks = [17, 40, 23]
    X = [rng.standard_normal((M, k)) for k in Ks]       # X_p: M x K_p
    Y = [rng.standard_normal((k, N)) for k in Ks]       # Y_p: K_p x N
    pb = [0, 2, 3, 3]                                   # pairs of C blocks 0, 1, 2
    for call, scale in enumerate((1.0, -0.5)):
        xs, ys = [scale * x for x in X], [y for y in Y]
        xflat, xo, ldx = _pack(xs, xt, pad=3)
        yflat, yo, ldy = _pack(ys, yt, pad=1)
        dX, dY = sb.DenseTensor(xflat, ctx=ctx), sb.DenseTensor(yflat, ctx=ctx)
        out = sb.DenseTensor(np.full(3 * M * N, np.nan), ctx=ctx)
        st, msg = _call(ctx._lib, ctx.stream, dX.device_ptr()[0], dY.device_ptr()[0], out.device_ptr()[0],
                        [0, M * N, 2 * M * N], [M] * 3, [N] * 3, pb, xo, yo, Ks, ldx, ldy, xt, yt)
        assert st == 0, msg
        ctx.synchronize()
        got = out.to_numpy().reshape(3, N, M).transpose(0, 2, 1)  # column-major blocks
        # the oracle's block products (contract_shared! sums the pairs of a C block in order)
        want = [_pairs_sum([(xs[0], ys[0]), (xs[1], ys[1])]), _pairs_sum([(xs[2], ys[2])]), np.zeros((M, N))]
        for c in range(3):
            ref = want[c]
            assert np.linalg.norm(got[c] - ref) <= RTOL * max(np.linalg.norm(ref), 1.0), (call, c)


def test_noalloc_rejects_plans_beyond_the_scratch_limit():
    import sparsebackends_b200 as sb
    ctx = sb.Context(0)
    lib = ctx._lib
    n = 4097
    one = (C.c_int32 * n)(*([1] * n))
    err = C.create_string_buffer(256)
    st = lib.sb_block_gemm_f64_noalloc(C.c_void_p(ctx.stream), C.c_void_p(8), C.c_void_p(8), C.c_void_p(8), n,
                                       (C.c_int64 * n)(), one, one, (C.c_int32 * (n + 1))(), None, None, None, None,
                                       None, 0, 0, err, 256)
    assert st == 1  # SB_ERR_INVALID_ARG, before any device work
    assert b"4096" in err.value


def test_noalloc_rejects_bad_leading_dimensions_and_offsets():
    import sparsebackends_b200 as sb
    ctx = sb.Context(0)
    buf = sb.DenseTensor(np.zeros(64), ctx=ctx)
    p = buf.device_ptr()[0]
    # M = 4, N = 4, K = 4: ldx 3 < M (untransposed X)
    st, msg = _call(ctx._lib, ctx.stream, p, p, p, [0], [4], [4], [0, 1], [0], [0], [4], [3], [4], 0, 0)
    assert st == 1 and "ld" in msg
    # negative offset
    st, msg = _call(ctx._lib, ctx.stream, p, p, p, [0], [4], [4], [0, 1], [-4], [0], [4], [4], [4], 0, 0)
    assert st == 1 and "negative" in msg
