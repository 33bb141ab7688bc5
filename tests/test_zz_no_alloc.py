"""The allocation-free entry point sb_block_gemm_f64_noalloc.

It serves callers that cannot allocate device memory during a solve (a fixed
pool or budget, or a host runtime that owns the device and forbids cudaMalloc):
they hand in device buffers for inputs and outputs, and the plan goes into the
library's static device scratch array instead of allocated buffers.

Checked here through the C ABI against the existing entry point sb_contract
(same block-sparse contraction, contract_shared! semantics) on two calls in a
row with different shapes, within the GEMM tolerance the parity tests use
(1e-12 relative Frobenius per block); plus the size limit.  The file sorts
last so that a run stopping at the first failure has run everything else.
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


def _run_noalloc(sb, ctx, A_t, B_t, C_t, A, B, ckeys, plist, M, K, N):
    lib = ctx._lib
    xA, _ = A_t.device_ptr()
    yB, _ = B_t.device_ptr()
    dC, _ = C_t.device_ptr()
    blkA, blkB, blkC = M * K, K * N, M * N
    nc = len(ckeys)
    c_off = (C.c_int64 * nc)(*[c * blkC for c in range(nc)])
    rows = (C.c_int32 * nc)(*([M] * nc))
    cols = (C.c_int32 * nc)(*([N] * nc))
    pb, xo, yo = [0], [], []
    for pl in plist:
        for ia, ib in pl:
            xo.append(ia * blkA)
            yo.append(ib * blkB)
        pb.append(len(xo))
    npairs = len(xo)
    err = C.create_string_buffer(256)
    st = lib.sb_block_gemm_f64_noalloc(
        C.c_void_p(ctx.stream), C.c_void_p(xA), C.c_void_p(yB), C.c_void_p(dC), nc, c_off, rows, cols,
        (C.c_int32 * (nc + 1))(*pb), (C.c_int64 * max(npairs, 1))(*xo), (C.c_int64 * max(npairs, 1))(*yo),
        (C.c_int32 * max(npairs, 1))(*([K] * npairs)), (C.c_int32 * max(npairs, 1))(*([M] * npairs)),
        (C.c_int32 * max(npairs, 1))(*([K] * npairs)), 0, 0, err, 256)
    assert st == 0, err.value.decode()
    ctx.synchronize()


@pytest.mark.parametrize("repeat", [0])
def test_noalloc_matches_sb_contract_on_two_calls(repeat):
    import sparsebackends_b200 as sb
    ctx = sb.Context(0)
    shapes = [(1, 3, 4, 3, 37, 29, 21), (2, 2, 3, 2, 130, 17, 9)]  # (seed, I, Q, J, M, K, N)
    for seed, I, Q, J, M, K, N in shapes:
        A, B = _case(seed, I, Q, J, M, K, N)
        lA, lB, lC = ["i", "q", "m", "k"], ["j", "q", "k", "n"], ["i", "j", "m", "n"]
        A_t = sb.NewBlockSparseSorted(A.dims, 2, A.keys, A.ids, A.data, ctx=ctx)
        B_t = sb.NewBlockSparseSorted(B.dims, 2, B.keys, B.ids, B.data, ctx=ctx)
        # existing entry point
        C_ref = sb.NewBlockSparseSorted.empty((I, J, M, N), 2, ctx=ctx)
        sb.contract_(C_ref, lC, A_t, lA, B_t, lB)
        ckeys, plist = _plan(A, B, (I, J))
        assert C_ref.keys == ckeys
        # allocation-free entry point into a caller-provided output buffer
        out = sb.DenseTensor(ctx=ctx, dims=(max(len(ckeys) * M * N, 1),))
        _run_noalloc(sb, ctx, A_t, B_t, out, A, B, ckeys, plist, M, K, N)
        got = out.to_numpy()
        ref = C_ref.data
        blk = M * N
        for c in range(len(ckeys)):
            g, r = got[c * blk:(c + 1) * blk], ref[c * blk:(c + 1) * blk]
            assert np.linalg.norm(g - r) <= RTOL * max(np.linalg.norm(r), 1e-300)


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
