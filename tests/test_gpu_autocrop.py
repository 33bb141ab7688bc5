"""Zero padding cropped inside contract_shared! (BS x BS) on uniform operands.

The library scans the operands' nonzero extents, makes them consistent over
the matched block pairs, contracts the cropped (ragged) blocks and pads the
result back.  Checked here:

* with zero padding that differs between the two operands of a pair (so the
  extents must be harmonised), the result has the oracle's keys and blocks
  (1e-12) and equals the uncropped contraction (1e-12); the trace line shows
  the cropped path ran;
* operands without padding decline the cropped path: the result is
  bit-identical to the uncropped one;
* the two-site H_eff chain in the reference layout, small and at chi = 2048,
  agrees with the uncropped chain (1e-12); the psi*L and R*T3 steps are
  cropped.

SPARSEB_AUTO_CROP (read when a context is created): 0 off, 1 the default
(compute-heavy contractions only), 2 whenever cropping saves work.
"""
import os

import numpy as np
import pytest

from oracle import sparse_oracle as so

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _ctx(sb, mode, trace=False):
    saved = {k: os.environ.get(k) for k in ("SPARSEB_AUTO_CROP", "SPARSEB_TRACE")}
    os.environ["SPARSEB_AUTO_CROP"] = str(mode)
    os.environ["SPARSEB_TRACE"] = "1" if trace else "0"
    try:
        return sb.Context(0)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _padded_pair(rng, pad=True):
    """A[(q, i) | (m, k)] x B[(q, j) | (k, n)] -> C[(i, j) | (m, n)]; with
    ``pad`` every block keeps a random leading sub-block and is zero beyond,
    independently in A and B (so A's k extent differs from B's)."""
    Q, I, J, M, K, N = 3, 4, 3, 9, 8, 7
    ka = sorted({(int(rng.integers(1, Q + 1)), int(rng.integers(1, I + 1))) for _ in range(9)}, key=lambda x: x[::-1])
    kb = sorted({(int(rng.integers(1, Q + 1)), int(rng.integers(1, J + 1))) for _ in range(7)}, key=lambda x: x[::-1])

    def blocks(keys, d0, d1):
        out = []
        for _ in keys:
            b = rng.standard_normal((d0, d1))
            if pad:
                b[int(rng.integers(1, d0 + 1)):, :] = 0.0
                b[:, int(rng.integers(1, d1 + 1)):] = 0.0
            out.append(b.reshape(-1, order="F"))
        return np.concatenate(out)

    A = ((Q, I, M, K), ka, blocks(ka, M, K))
    B = ((Q, J, K, N), kb, blocks(kb, K, N))
    return A, B, (I, J, M, N)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_harmonised_crop_matches_oracle_and_uncropped(seed, capfd):
    import sparsebackends_b200 as sb
    rng = np.random.Generator(np.random.PCG64(seed))
    (da, ka, xa), (db, kb, xb), dc = _padded_pair(rng)
    lA, lB, lC = ["q", "i", "m", "k"], ["q", "j", "k", "n"], ["i", "j", "m", "n"]
    out = {}
    for mode in (0, 2):
        ctx = _ctx(sb, mode, trace=True)
        A = sb.NewBlockSparseSorted(da, 2, ka, None, xa, ctx=ctx)
        B = sb.NewBlockSparseSorted(db, 2, kb, None, xb, ctx=ctx)
        C = sb.NewBlockSparseSorted.empty(dc, 2, ctx=ctx)
        sb.contract_(C, lC, A, lA, B, lB)
        out[mode] = (C.keys, C.blocks_by_key(), C.is_ragged)
        err = capfd.readouterr().err
        assert ("zero padding cropped" in err) == (mode == 2), err
    ref = so.contract(so.BS.empty(dc, 2), lC, so.BS(da, 2, ka, list(range(1, len(ka) + 1)), xa), lA,
                      so.BS(db, 2, kb, list(range(1, len(kb) + 1)), xb), lB)
    rb = ref.blocks_by_key()
    for mode in (0, 2):
        keys, blocks, ragged = out[mode]
        assert not ragged
        assert keys == ref.keys
        for key in rb:
            assert _rel(blocks[key], np.ravel(rb[key], order="F")) <= RTOL
    for key in rb:
        assert _rel(out[2][1][key], out[0][1][key]) <= RTOL


def test_unpadded_operands_decline(capfd):
    import sparsebackends_b200 as sb
    rng = np.random.Generator(np.random.PCG64(9))
    (da, ka, xa), (db, kb, xb), dc = _padded_pair(rng, pad=False)
    lA, lB, lC = ["q", "i", "m", "k"], ["q", "j", "k", "n"], ["i", "j", "m", "n"]
    got = {}
    for mode in (0, 2):
        ctx = _ctx(sb, mode, trace=True)
        A = sb.NewBlockSparseSorted(da, 2, ka, None, xa, ctx=ctx)
        B = sb.NewBlockSparseSorted(db, 2, kb, None, xb, ctx=ctx)
        C = sb.NewBlockSparseSorted.empty(dc, 2, ctx=ctx)
        sb.contract_(C, lC, A, lA, B, lB)
        got[mode] = (C.keys, np.array(C.data, copy=True))
        assert "zero padding cropped" not in capfd.readouterr().err
    assert got[0][0] == got[2][0] and np.array_equal(got[0][1], got[2][1])


def _uniform_chain(sb, qn, lay, host, mode):
    ctx = _ctx(sb, mode)
    dev = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx) for n, (k, d) in host.items()}
    out = qn.HeffChain(lay, ctx).apply(dev["psi"], dev["L"], dev["W1"], dev["W2"], dev["R"])
    return out.keys, np.array(out.data, copy=True), out.is_ragged


def test_small_heff_chain_forced(capfd):
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    from tests.heff_dense import small_layout
    lay = small_layout(48)
    rng = np.random.Generator(np.random.PCG64(4))
    host = {n: qn.random_block_tensor(lay, n, rng, 0.5) for n in ("psi", "L", "W1", "W2", "R")}
    k0, d0, r0 = _uniform_chain(sb, qn, lay, host, 0)
    ctx = _ctx(sb, 2, trace=True)
    dev = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx) for n, (k, d) in host.items()}
    out = qn.HeffChain(lay, ctx).apply(dev["psi"], dev["L"], dev["W1"], dev["W2"], dev["R"])
    lines = [ln for ln in capfd.readouterr().err.splitlines() if "contract_shared" in ln]
    assert len(lines) == 4 and all("zero padding cropped" in ln for ln in lines), lines
    assert not out.is_ragged and not r0 and out.keys == k0
    assert _rel(out.data, d0) <= RTOL


def test_full_size_reference_layout_chain():
    import time

    import bench
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    lay = bench.workload(2048)
    host = bench.host_tensors(lay, 2026)
    res = {}
    for mode in (0, 1):
        t0 = time.perf_counter()
        res[mode] = _uniform_chain(sb, qn, lay, host, mode)
        print(f"auto_crop={mode}: {time.perf_counter() - t0:.2f} s (with uploads)")
    assert res[0][0] == res[1][0]
    assert _rel(res[1][1], res[0][1]) <= RTOL
