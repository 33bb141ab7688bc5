"""sb_tensor_crop_padding: operands in the reference's zero-padded layout
cropped, from their values, to the smallest block extents that keep every
nonzero entry.  On U(1) H_eff operands (random sector blocks) that recovers
the sector extents exactly, so the chain on the cropped operands is the ragged
chain bit for bit; the padded chain agrees to 1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as sbmod
    return sbmod


def _pack(blocks):
    return np.concatenate([b.reshape(-1, order="F") for b in blocks]) if blocks else np.zeros(0)


def test_edge_cases(sb):
    """All-zero blocks keep extent 1; a lone nonzero fixes each axis extent;
    a ragged input is cropped further; the result pads back to the input."""
    rng = np.random.Generator(np.random.PCG64(1))
    dims = (3, 5, 4, 6)  # prefix 1 axis, tail (5, 4, 6) -> n2 = 3
    blocks = [np.zeros((5, 4, 6)), np.zeros((5, 4, 6)), rng.standard_normal((5, 4, 6))]
    blocks[1][2, 0, 3] = 7.0
    blocks[2][4:, :, :] = 0.0
    blocks[2][:, :, 5] = 0.0
    keys = [(1,), (2,), (3,)]
    A = sb.NewBlockSparseSorted(dims[:1] + (5, 4, 6), 3, keys, None, _pack(blocks))
    R = sb.crop_padding(A)
    assert R.keys == keys
    assert R.block_dims == [(1, 1, 1), (3, 1, 4), (4, 4, 5)]
    assert np.array_equal(sb.to_dense(sb.to_uniform(R)), sb.to_dense(A))
    # ragged input: block 3 at (4, 4, 5) already; zero its last k-slice too
    b3 = blocks[2][:4, :, :5].copy()
    b3[:, 3, :] = 0.0
    Rg = sb.NewBlockSparseSorted(A.dims, 3, keys, None, _pack([blocks[0][:1, :1, :1], blocks[1][:3, :1, :4], b3]),
                                 block_dims=[(1, 1, 1), (3, 1, 4), (4, 4, 5)])
    assert sb.crop_padding(Rg).block_dims == [(1, 1, 1), (3, 1, 4), (4, 3, 5)]
    # no blocks at all
    E = sb.NewBlockSparseSorted.empty((3, 5, 4, 6), 3)
    assert sb.crop_padding(E).keys == []


def test_heff_operands_recover_sector_extents(sb):
    from sparsebackends_b200 import qn
    from tests.heff_dense import small_layout
    lay = small_layout(48)
    rng = np.random.Generator(np.random.PCG64(2))
    ops = qn.hermitian_operators(lay, rng)
    ops["psi"] = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    ctx = sb.Context(0)
    rag, pad, crop = {}, {}, {}
    for n, (k, d, e) in ops.items():
        rag[n] = sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx, block_dims=e)
        pad[n] = sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, qn.pad_ragged(lay, n, k, d, e), ctx=ctx)
        crop[n] = sb.crop_padding(pad[n])
        assert crop[n].keys == rag[n].keys
        assert crop[n].block_dims == [tuple(x) for x in e], n
        assert np.array_equal(crop[n].data, rag[n].data), n
    outs = {}
    for name, T in (("ragged", rag), ("cropped", crop), ("padded", pad)):
        chain = qn.HeffChain(lay, ctx)
        out = chain.apply(T["psi"], T["L"], T["W1"], T["W2"], T["R"])
        outs[name] = sb.to_uniform(out) if out.is_ragged else out
        outs[name] = (outs[name].keys, np.array(outs[name].data, copy=True))
    assert outs["cropped"][0] == outs["ragged"][0] and np.array_equal(outs["cropped"][1], outs["ragged"][1])
    assert outs["padded"][0] == outs["ragged"][0]
    a, b = outs["ragged"][1], outs["padded"][1]
    assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)


def test_full_size_operands(sb):
    """The chi = 2048 benchmark operands in the padded layout crop to exactly
    their sector extents."""
    import bench
    lay = bench.workload(2048)
    host, host_r = bench.host_tensors(lay, 2026, with_ragged=True)
    ctx = sb.Context(0)
    for n in ("psi", "L", "W1"):
        keys, data = host[n]
        _, rdata, exts = host_r[n]
        P = sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], keys, None, data, ctx=ctx)
        R = sb.crop_padding(P)
        assert R.block_dims == [tuple(x) for x in exts], n
        assert np.array_equal(R.data, rdata), n
