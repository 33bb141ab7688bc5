"""CPU checks of the U(1) two-site split (``qn.split_two_site``), the SVD step
of a two-site DMRG update on the block format:

* without truncation A·B reproduces every block of ψ (1e-12);
* A is left-orthonormal per bond sector (absorb="right"), or B is
  right-orthonormal (absorb="left");
* ``maxdim`` keeps that many singular values in all, the largest ones, and
  the squared reconstruction error equals the reported dropped weight;
* ``cutoff`` drops the smallest values while the dropped weight stays within
  cutoff · Σ s², and no further one could be dropped;
* the dense ground-state energies that the DMRG tests compare with match
  closed forms.
"""
import numpy as np
import pytest

from sparsebackends_b200 import qn
from tests.heff_dense import small_layout


def _psi(seed, chi=24):
    lay = small_layout(chi)
    rng = np.random.Generator(np.random.PCG64(seed))
    keys, data, exts = qn.random_block_tensor(lay, "psi", rng, 1.0, ragged=True)
    return lay, keys, data, exts


def _blocks(keys, data, exts):
    out, off = {}, 0
    for k, e in zip(keys, exts):
        n = int(np.prod(e))
        out[tuple(k)] = data[off: off + n].reshape(e, order="F")
        off += n
    return out


def _rebuild(lay, A, B, link):
    a, b = _blocks(*A), _blocks(*B)
    out = {}
    for (ql, s1, qc), x in a.items():
        for (qc2, s2, qr), y in b.items():
            if qc2 == qc:
                k = (ql, s1, s2, qr)
                out[k] = out.get(k, 0) + x @ y
    return out


@pytest.mark.parametrize("absorb", ["right", "left"])
@pytest.mark.parametrize("seed", [0, 1])
def test_exact_split_and_orthonormality(absorb, seed):
    lay, keys, data, exts = _psi(seed)
    A, B, link, sv, err = qn.split_two_site(lay, keys, data, exts, absorb=absorb)
    assert err == pytest.approx(0.0, abs=1e-20)
    psi = _blocks(keys, data, exts)
    rec = _rebuild(lay, A, B, link)
    for k, blk in psi.items():
        assert np.linalg.norm(rec[k] - blk) <= 1e-12 * np.linalg.norm(blk)
    # sector dims of the new bond are the ranks of the charge blocks
    assert sum(link.dims) == len(sv)
    side = _blocks(*A) if absorb == "right" else _blocks(*B)
    for qc in range(1, link.S + 1):
        if absorb == "right":
            G = sum(x.T @ x for (ql, s1, q), x in side.items() if q == qc)
        else:
            G = sum(x @ x.T for (q, s2, qr), x in side.items() if q == qc)
        assert np.allclose(G, np.eye(link.dims[qc - 1]), atol=1e-12)
    # keys column-major sorted, extents consistent with the links
    for (ks, _, es), (lft, rgt) in ((A, (lay.left, link)), (B, (link, lay.right))):
        assert ks == sorted(ks, key=lambda k: k[::-1])
        for k, e in zip(ks, es):
            assert e == (lft.dims[k[0] - 1], rgt.dims[k[2] - 1])


def test_maxdim_truncation_error():
    lay, keys, data, exts = _psi(3)
    _, _, _, sv_all, _ = qn.split_two_site(lay, keys, data, exts)
    m = 10
    A, B, link, sv, err = qn.split_two_site(lay, keys, data, exts, maxdim=m)
    assert len(sv) == sum(link.dims) == m
    assert np.allclose(sv, np.sort(sv_all)[::-1][:m])
    assert err == pytest.approx(float(np.sum(np.sort(sv_all)[::-1][m:] ** 2)), rel=1e-12)
    psi = _blocks(keys, data, exts)
    rec = _rebuild(lay, A, B, link)
    e2 = sum(np.linalg.norm(rec.get(k, 0) - blk) ** 2 for k, blk in psi.items())
    assert e2 == pytest.approx(err, rel=1e-8)


def test_cutoff_rule():
    lay, keys, data, exts = _psi(4)
    _, _, _, sv_all, _ = qn.split_two_site(lay, keys, data, exts)
    w = np.sort(sv_all)[::-1] ** 2
    total = w.sum()
    cut = 0.05
    _, _, link, sv, err = qn.split_two_site(lay, keys, data, exts, cutoff=cut)
    m = len(sv)
    assert err <= cut * total + 1e-15
    assert m == 1 or w[m - 1:].sum() > cut * total  # one more drop would exceed the cutoff


def test_exact_diagonalisation_reference_energies():
    """The dense reference of the DMRG tests against closed forms: the
    two-site singlet (-3/4), four sites (-(3 + 2 sqrt 3)/4), and the XX chain
    (Delta = 0), free fermions with single-particle energies cos(k pi/(N+1))
    filled up to half filling."""
    from sparsebackends_b200 import dmrg
    assert dmrg.exact_ground_energy(2) == pytest.approx(-0.75, abs=1e-13)
    assert dmrg.exact_ground_energy(4) == pytest.approx(-(3 + 2 * np.sqrt(3)) / 4, abs=1e-12)
    n = 8
    eps = np.sort(np.cos(np.arange(1, n + 1) * np.pi / (n + 1)))
    assert dmrg.exact_ground_energy(n, 0.0) == pytest.approx(eps[: n // 2].sum(), abs=1e-12)
