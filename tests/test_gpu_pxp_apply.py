"""The PXP chain's MPO applied to an MPS site tensor at its benchmark shapes
(H = sum_i P_{i-1} X_i P_{i+1}, P = |0><0|; MPO bond 4 with 5 of 16 nonzero
(wl, wr) blocks, 8 nonzeros; site tensor chi = 256, d = 2), with the MPO in the
two sparse storages the reference uses for it, against the oracle:

* COO x Dense -> block-sparse (contract!, ta/contract_coo_dense.jl:4-125): one
  65536-element block per nonzero, values bit-exact (scaled adds with the
  reference's rounding);
* COO x block-sparse, the site tensor's physical index in the prefix
  (contract_prefix!, ta/contract_coo_bs.jl): bit-exact;
* COO x Dense -> aliased (contract_aliased!, ta/contract_aliased_coo_dense.jl:
  34-164): one template per physical index value, scalars per key.
"""
import numpy as np
import pytest

from oracle import sparse_oracle as so
from tests.test_gpu_parity import assert_aliased_equal, assert_bs_equal, lib_empty_like, lib_operand

pytestmark = pytest.mark.gpu

CHI, D, W = 256, 2, 4


def pxp_mpo():
    """W[s', s, wl, wr]: channels 1 = identity before, 2 = P placed, 3 = P X
    placed, 4 = identity after (lower-triangular bond-4 MPO)."""
    I = np.eye(D)
    P = np.array([[1.0, 0.0], [0.0, 0.0]])
    X = np.array([[0.0, 1.0], [1.0, 0.0]])
    Wd = np.zeros((D, D, W, W))
    for (wl, wr), op in {(0, 0): I, (1, 0): P, (2, 1): X, (3, 2): P, (3, 3): I}.items():
        Wd[:, :, wl, wr] = op
    return Wd


@pytest.fixture(scope="module")
def sb():
    import sparsebackends_b200 as sbmod
    return sbmod


@pytest.fixture(scope="module")
def operands():
    rng = np.random.Generator(np.random.PCG64(64))
    Wd = pxp_mpo()
    Wc = so.coo_from_dense(Wd, atol=0.0)
    assert len(Wc.keys) == 8
    psi = rng.standard_normal((CHI, D, CHI))
    return Wd, Wc, psi


def test_coo_dense_to_blocksparse(sb, operands):
    Wd, Wc, psi = operands
    lW, lpsi, lC = ["sp", "s", "wl", "wr"], ["l", "s", "r"], ["sp", "wl", "wr", "l", "r"]
    C0 = so.BS.empty((D, W, W, CHI, CHI), 2)
    Cref = so.contract(C0, lC, Wc, lW, psi, lpsi)
    Cg = lib_empty_like(sb, C0)
    sb.contract_(Cg, lC, lib_operand(sb, Wc), lW, lib_operand(sb, psi), lpsi)
    assert len(Cref.keys) == 8
    assert_bs_equal(Cg, Cref, exact=True)
    want = np.einsum("pswv,lsr->pwvlr", Wd, psi)
    assert np.array_equal(sb.to_dense(Cg), want)


def test_coo_blocksparse_prefix(sb, operands):
    Wd, Wc, psi = operands
    psi_bs = so.blocksparse_from_dense(np.ascontiguousarray(psi.transpose(1, 0, 2)), 2)  # (s | l, r)
    lW, lpsi, lC = ["sp", "s", "wl", "wr"], ["s", "l", "r"], ["sp", "wl", "wr", "l", "r"]
    C0 = so.BS.empty((D, W, W, CHI, CHI), 2)
    Cref = so.contract(C0, lC, Wc, lW, psi_bs, lpsi)
    Cg = lib_empty_like(sb, C0)
    sb.contract_(Cg, lC, lib_operand(sb, Wc), lW, lib_operand(sb, psi_bs), lpsi)
    assert_bs_equal(Cg, Cref, exact=True)
    assert np.array_equal(sb.to_dense(Cg), np.einsum("pswv,lsr->pwvlr", Wd, psi))


def test_coo_dense_to_aliased(sb, operands):
    Wd, Wc, psi = operands
    lW, lpsi, lC = ["sp", "s", "wl", "wr"], ["l", "s", "r"], ["sp", "wl", "wr", "l", "r"]
    C0 = so.Aliased.empty((D, W, W, CHI, CHI), 2)
    Cref = so.contract(C0, lC, Wc, lW, psi, lpsi)
    Cg = lib_empty_like(sb, C0)
    sb.contract_(Cg, lC, lib_operand(sb, Wc), lW, lib_operand(sb, psi), lpsi)
    assert_aliased_equal(Cg, Cref)
    blocks = Cg.logical_blocks()
    want = np.einsum("pswv,lsr->pwvlr", Wd, psi)
    for k, v in blocks.items():
        assert np.array_equal(np.asarray(v).reshape(-1, order="F"),
                              want[k[0] - 1, k[1] - 1, k[2] - 1].reshape(-1, order="F")), k
