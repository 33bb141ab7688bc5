"""GPU environment updates (ITensorMPS makeL!/makeR!) on the contract! kernels.

L' = L·A·W·Ā and R' = R·B·W·B̄ through three BS×BS contract! calls each,
against dense einsums of the same seeded U(1)-structured blocks (1e-12
relative Frobenius): uniform (zero-padded) and ragged layouts.
"""
import numpy as np
import pytest

from sparsebackends_b200 import qn

pytestmark = pytest.mark.gpu


def _layout():
    left = qn.gaussian_sectors(20, [-4, -2, 0, 2, 4], width=1.5)
    right = qn.gaussian_sectors(22, [-5, -3, -1, 1, 3, 5], width=1.8)
    return qn.HeffLayout(left, right, qn.mpo_link({-2: 2, 0: 3, 2: 2}))


def _offsets(link):
    return np.concatenate([[0], np.cumsum(link.dims)[:-1]]).astype(int)


def _dense(lay, kind, keys, data, exts, links):
    """Dense array of a tensor whose prefix axes map to `links` (one entry per
    prefix axis: a U1Link or an int for a plain axis such as the spin)."""
    shape = [l.total if isinstance(l, qn.U1Link) else l for l in links]
    out = np.zeros(shape)
    offs = [(_offsets(l) if isinstance(l, qn.U1Link) else None) for l in links]
    off = 0
    for k, e in zip(keys, exts):
        cnt = int(np.prod(e))
        blk = data[off: off + cnt].reshape(e, order="F")
        off += cnt
        idx, t = [], 0
        full = []
        for a, l in enumerate(links):
            if isinstance(l, qn.U1Link):
                full.append(slice(offs[a][k[a] - 1], offs[a][k[a] - 1] + e[t]))
                t += 1
            else:
                full.append(k[a] - 1)
        out[tuple(full)] = blk
    return out


def _tensors(ragged, seed):
    import sparsebackends_b200 as sb
    lay = _layout()
    rng = np.random.Generator(np.random.PCG64(seed))
    host = {n: qn.random_block_tensor(lay, n, rng, 0.5, ragged=True) for n in ("L", "R", "W1", "A")}
    ctx = sb.Context(0)
    dev = {}
    for n, (k, d, e) in host.items():
        if ragged:
            dev[n] = sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx, block_dims=e)
        else:
            dev[n] = sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, qn.pad_ragged(lay, n, k, d, e), ctx=ctx)
    w = lay.mpo
    # L/R: (q', qw, q) with the channel link in the middle; the tails follow the prefix order
    dense = {
        "L": _dense(lay, "L", *host["L"], [lay.left, w, lay.left]),
        "R": _dense(lay, "R", *host["R"], [lay.right, w, lay.right]),
        "W": _dense(lay, "W1", *host["W1"], [w, 2, 2, w]),
        "A": _dense(lay, "A", *host["A"], [lay.left, 2, lay.right]),
    }
    return sb, lay, dev, dense


def _check(got, want):
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)


@pytest.mark.parametrize("ragged", [False, True])
def test_make_L_matches_dense(ragged):
    sb, lay, dev, d = _tensors(ragged, 31)
    Ln = qn.make_L(dev["L"], dev["A"], dev["W1"])
    want = np.einsum("xwa,asb,wtsv,xty->yvb", d["L"], d["A"], d["W"], d["A"])
    Ld = sb.to_dense(sb.to_uniform(Ln) if ragged else Ln)
    # uniform dense layout: (S_r, S_w, S_r, D_r, D_w, D_r) -> global (y, v, b)
    _check(_pad_to_global(Ld, lay.right, lay.mpo, lay.right), want)


@pytest.mark.parametrize("ragged", [False, True])
def test_make_R_matches_dense(ragged):
    sb, lay, dev, d = _tensors(ragged, 32)
    # B = A on the left/right links; R over the right link
    Rn = qn.make_R(dev["R"], dev["A"], dev["W1"])
    want = np.einsum("ywb,asb,vtsw,xty->xva", d["R"], d["A"], d["W"], d["A"])
    Rd = sb.to_dense(sb.to_uniform(Rn) if ragged else Rn)
    _check(_pad_to_global(Rd, lay.left, lay.mpo, lay.left), want)


def _pad_to_global(D, l1, l2, l3):
    """(S1, S2, S3, D1, D2, D3) sector-padded dense -> (tot1, tot2, tot3)."""
    out = np.zeros((l1.total, l2.total, l3.total))
    o1, o2, o3 = _offsets(l1), _offsets(l2), _offsets(l3)
    for a in range(l1.S):
        for b in range(l2.S):
            for c in range(l3.S):
                out[o1[a]:o1[a] + l1.dims[a], o2[b]:o2[b] + l2.dims[b], o3[c]:o3[c] + l3.dims[c]] = \
                    D[a, b, c, :l1.dims[a], :l2.dims[b], :l3.dims[c]]
    return out
