"""The plan cache of contract_shared! (BS x BS): a contraction whose labels and
operand block structure (dims, tail count, keys, block extents) equal a recent
one reuses its output layout and prepared GEMM.  Reuse must be invisible in
the results: bit-identical to a context without the cache
(SPARSEB_PLAN_CACHE=0), for new operand values on the same structure, and a
changed structure must not be served from the cache.
"""
import contextlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def _env(**kv):
    old = {k: os.environ.get(k) for k in kv}
    os.environ.update({k: str(v) for k, v in kv.items()})
    try:
        yield
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _ctx(sb, **kv):
    with _env(SPARSEB_TRACE=1, **kv):
        return sb.Context(0)


def _ragged_pair(sb, ctx, rng, ms, ks, ns, drop=None):
    """A[(i, q) | m, k] and B[(j, q) | k, n] with per-block extents."""
    Akeys = [(i + 1, q + 1) for q in range(len(ks)) for i in range(len(ms)) if (i + 1, q + 1) != drop]
    Bkeys = [(j + 1, q + 1) for q in range(len(ks)) for j in range(len(ns))]
    Ab = {k: rng.standard_normal((ms[k[0] - 1], ks[k[1] - 1])) for k in Akeys}
    Bb = {k: rng.standard_normal((ks[k[1] - 1], ns[k[0] - 1])) for k in Bkeys}

    def tensor(keys, blocks, dims):
        data = np.concatenate([blocks[k].reshape(-1, order="F") for k in keys])
        return sb.NewBlockSparseSorted(dims, 2, keys, None, data, ctx=ctx, block_dims=[blocks[k].shape for k in keys])

    return (tensor(Akeys, Ab, (len(ms), len(ks), max(ms), max(ks))),
            tensor(Bkeys, Bb, (len(ns), len(ks), max(ks), max(ns))))


LAB = (["i", "j", "m", "n"], ["i", "q", "m", "k"], ["j", "q", "k", "n"])
MS, KS, NS = [18, 133, 64, 100], [40, 250, 7], [411, 20, 70]


def _contract(sb, ctx, A, B):
    C = sb.NewBlockSparseSorted.empty((A.dims[0], B.dims[0], A.dims[2], B.dims[3]), 2, ctx=ctx)
    sb.contract_(C, LAB[0], A, LAB[1], B, LAB[2])
    return C.keys, np.array(C.data, copy=True), C.block_dims


def test_repeat_is_cached_and_bit_identical(sb_mod, capfd):
    sb = sb_mod
    on, off = _ctx(sb), _ctx(sb, SPARSEB_PLAN_CACHE=0)
    got = []
    for seed in (1, 1, 2):  # same structure: the same values twice, then new values
        rng = np.random.Generator(np.random.PCG64(seed))
        A, B = _ragged_pair(sb, on, rng, MS, KS, NS)
        r_on = _contract(sb, on, A, B)
        tr = capfd.readouterr().err
        rng = np.random.Generator(np.random.PCG64(seed))
        A2, B2 = _ragged_pair(sb, off, rng, MS, KS, NS)
        r_off = _contract(sb, off, A2, B2)
        capfd.readouterr()
        assert r_on[0] == r_off[0] and r_on[2] == r_off[2]
        assert np.array_equal(r_on[1], r_off[1])
        got.append(("(cached plan)" in tr, r_on))
    assert [c for c, _ in got] == [False, True, True]
    assert np.array_equal(got[0][1][1], got[1][1][1])


def test_changed_structure_is_not_served_from_cache(sb_mod, capfd):
    sb = sb_mod
    on, off = _ctx(sb), _ctx(sb, SPARSEB_PLAN_CACHE=0)
    rng = np.random.Generator(np.random.PCG64(3))
    _contract(sb, on, *_ragged_pair(sb, on, rng, MS, KS, NS))
    capfd.readouterr()
    for kw in ({"drop": (2, 1)}, {}, {"ms": [18, 133, 64, 99]}):  # a block less; back; other extents
        ms = kw.pop("ms", MS)
        rng = np.random.Generator(np.random.PCG64(4))
        r_on = _contract(sb, on, *_ragged_pair(sb, on, rng, ms, KS, NS, **kw))
        tr = capfd.readouterr().err
        rng = np.random.Generator(np.random.PCG64(4))
        r_off = _contract(sb, off, *_ragged_pair(sb, off, rng, ms, KS, NS, **kw))
        capfd.readouterr()
        assert r_on[0] == r_off[0] and r_on[2] == r_off[2] and np.array_equal(r_on[1], r_off[1])
        assert ("(cached plan)" in tr) == (not kw and ms == MS), (kw, tr)


def test_heff_chain_and_eviction(sb_mod, capfd):
    """Repeated H_eff applies are served from the cache after the first; more
    structures than the cache holds evict the oldest without harm."""
    sb = sb_mod
    from sparsebackends_b200 import qn
    from tests.heff_dense import small_layout
    lay = small_layout(48)
    rng = np.random.Generator(np.random.PCG64(5))
    ops = qn.hermitian_operators(lay, rng)
    pk, pd, pe = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    outs = []
    for flag in (1, 0):
        ctx = _ctx(sb, SPARSEB_PLAN_CACHE=flag)
        T = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx, block_dims=e)
             for n, (k, d, e) in ops.items()}
        psi = sb.NewBlockSparseSorted(lay.dims["psi"], lay.n2["psi"], pk, None, pd, ctx=ctx, block_dims=pe)
        chain = qn.HeffChain(lay, ctx)
        res = []
        for _ in range(3):
            res.append(np.array(chain.apply(psi, T["L"], T["W1"], T["W2"], T["R"]).data, copy=True))
        tr = capfd.readouterr().err
        if flag:
            lines = [l for l in tr.splitlines() if l.startswith("[sparseb]")]
            assert len(lines) == 12 and sum("(cached plan)" in l for l in lines) == 8, tr
        outs.append(res)
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    # 40 distinct structures through one context (the cache holds 32), then the first again
    ctx = _ctx(sb)
    rng = np.random.Generator(np.random.PCG64(6))
    first = None
    for t in range(41):
        ms = [18 + (t % 40), 133, 64, 100]
        r = _contract(sb, ctx, *_ragged_pair(sb, ctx, np.random.Generator(np.random.PCG64(7)), ms, KS, NS))
        if t == 0:
            first = r
    capfd.readouterr()
    assert r[0] == first[0] and np.array_equal(r[1], first[1])


@pytest.fixture(scope="module")
def sb_mod():
    import sparsebackends_b200 as sb
    return sb


def test_autotuned_gemm_matches_oracle(monkeypatch):
    """SPARSEB_AUTOTUNE=1: the first launch of a block-shape histogram times the
    tile shapes and keeps the fastest; results stay within the drop-in
    tolerance, a second call (same histogram) reuses the choice, and repeated
    calls are bit-identical."""
    import numpy as np
    import sparsebackends_b200 as sb
    from oracle import sparse_oracle as so
    monkeypatch.setenv("SPARSEB_AUTOTUNE", "1")
    ctx = sb.Context(0)
    rng = np.random.Generator(np.random.PCG64(19))
    A = so.blocksparse_from_dense(rng.standard_normal((2, 3, 200, 150)), 2)
    B = so.blocksparse_from_dense(rng.standard_normal((3, 2, 150, 90)), 2)
    lC, lA, lB = ["i", "j", "m", "n"], ["i", "q", "m", "k"], ["q", "j", "k", "n"]
    ref = so.contract(so.BS.empty((2, 2, 200, 90), 2), lC, A, lA, B, lB)
    a = sb.NewBlockSparseSorted(A.dims, 2, A.keys, A.ids, A.data, ctx=ctx)
    b = sb.NewBlockSparseSorted(B.dims, 2, B.keys, B.ids, B.data, ctx=ctx)
    outs = []
    for _ in range(3):
        C = sb.NewBlockSparseSorted.empty((2, 2, 200, 90), 2, ctx=ctx)
        sb.contract_(C, lC, a, lA, b, lB)
        outs.append(np.array(C.data, copy=True))
        assert C.keys == ref.keys
        gb = C.blocks_by_key()
        for k, v in ref.blocks_by_key().items():
            assert np.linalg.norm(np.asarray(gb[k]) - v) <= 1e-12 * np.linalg.norm(v)
    assert np.array_equal(outs[1], outs[2])
