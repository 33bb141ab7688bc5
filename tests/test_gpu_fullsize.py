"""The benchmark workload at its full size (two-site H_eff, U(1), chi = 2048,
MPO link of 38 channels, 2.3 GB intermediates).

Against the CPU oracle (one matvec, about 20 s on 8 host BLAS threads):
the GPU chain's output key list equals the oracle's, and every block agrees
to 1e-12 relative Frobenius error (FP64 path) or 2e-5 (3xTF32 tensor-core path
with FP32 intermediates), on the reference's zero-padded layout.

Through properties that hold at any size:

* the output key list is exactly the one the key-level simulation of the four
  contractions predicts (integer work: bit-exact), and every ragged block has
  its sector extents;
* H_eff is linear: H(psi1 + 2 psi2) = H psi1 + 2 H psi2 (1e-12 relative);
* the ragged and the zero-padded (reference layout) chains agree (1e-12);
* repeated applies are bit-identical (no atomics, fixed accumulation order);
* the device norm of the result equals the host norm of its entries (1e-13).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHI = 2048


@pytest.fixture(scope="module")
def setup():
    import bench
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    lay = bench.workload(CHI)
    host, host_r = bench.host_tensors(lay, 2026, with_ragged=True)
    ctx = sb.Context(0)
    dev = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx, block_dims=e)
           for n, (k, d, e) in host_r.items()}
    chain = qn.HeffChain(lay, ctx)
    return sb, qn, lay, host, host_r, ctx, dev, chain


def _apply(setup, psi):
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    out = chain.apply(psi, dev["L"], dev["W1"], dev["W2"], dev["R"])
    return out.keys, np.array(out.data, copy=True), out


def _psi(setup, data):
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    keys, _, exts = host_r["psi"]
    return sb.NewBlockSparseSorted(lay.dims["psi"], lay.n2["psi"], keys, None, data, ctx=ctx, block_dims=exts)


def test_output_keys_and_extents(setup):
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    keys, data, out = _apply(setup, dev["psi"])
    lc = lay.labels["T4"]
    pc = len(lc) - lay.n2["T4"]
    want = {tuple(kv[x] for x in lc[:pc]) for kv in qn.chain_structure(lay)[-1]["pairs"]}
    # column-major order of the prefix keys: the last axis varies slowest
    assert keys == sorted(want, key=lambda k: k[::-1])
    # the tail axes of T4 are the MPS link intra-sector axes (ml, mr order of
    # the labels), each block at its sectors' extents
    ext = {x: qn._link_of(lay, qn.GRADE[x]) for x in lc[pc:]}
    grade_pos = {qn.GRADE[x]: lc.index(qn.GRADE[x]) for x in lc[pc:]}
    bd = out.block_dims
    for k, e in zip(keys, bd):
        assert tuple(e) == tuple(ext[x].dims[k[grade_pos[qn.GRADE[x]]] - 1] for x in lc[pc:])
    assert data.size == sum(int(np.prod(e)) for e in bd)


def test_linearity(setup):
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    _, d1, _ = host_r["psi"]
    d2 = np.random.Generator(np.random.PCG64(77)).standard_normal(d1.size)
    k1, h1, _ = _apply(setup, _psi(setup, d1))
    k2, h2, _ = _apply(setup, _psi(setup, d2))
    k3, h3, _ = _apply(setup, _psi(setup, d1 + 2.0 * d2))
    assert k1 == k2 == k3
    want = h1 + 2.0 * h2
    assert np.linalg.norm(h3 - want) <= 1e-12 * np.linalg.norm(want)


def test_ragged_equals_uniform_and_repeats_bit_identical(setup):
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    keys, a, out = _apply(setup, dev["psi"])
    ur = sb.to_uniform(out)
    ur_keys, ur_data = ur.keys, np.array(ur.data, copy=True)
    _, b, _ = _apply(setup, dev["psi"])
    assert np.array_equal(a, b)
    dev_u = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=ctx) for n, (k, d) in host.items()}
    chain_u = qn.HeffChain(lay, ctx)
    outu = chain_u.apply(dev_u["psi"], dev_u["L"], dev_u["W1"], dev_u["W2"], dev_u["R"])
    assert outu.keys == ur_keys
    du = np.array(outu.data, copy=True)
    assert np.linalg.norm(ur_data - du) <= 1e-12 * np.linalg.norm(du)


def test_device_norm(setup):
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    _, data, out = _apply(setup, dev["psi"])
    assert abs(sb.norm(out) - np.linalg.norm(data)) <= 1e-13 * np.linalg.norm(data)


@pytest.fixture(scope="module")
def oracle_t4(setup):
    """The oracle's four-step chain on the zero-padded operands."""
    from oracle import sparse_oracle as so
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    t = {n: so.BS(lay.dims[n], lay.n2[n], k, list(range(1, len(k) + 1)), d) for n, (k, d) in host.items()}
    lab = lay.labels
    for c, a, b in qn.HeffChain.STEPS:
        t[c] = so.contract(so.BS.empty(lay.dims[c], lay.n2[c]), lab[c], t[a], lab[a], t[b], lab[b])
    return t["T4"]


def _against_oracle(sb, out, ref, tol):
    got = sb.to_uniform(out)
    assert got.keys == ref.keys
    gb, rb = got.blocks_by_key(), ref.blocks_by_key()
    worst = 0.0
    for k, v in rb.items():
        e = float(np.linalg.norm(gb[k] - v) / max(np.linalg.norm(v), 1e-300))
        worst = max(worst, e)
        assert e <= tol, (k, e)
    return worst


def test_full_size_matches_oracle(setup, oracle_t4):
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    out = chain.apply(dev["psi"], dev["L"], dev["W1"], dev["W2"], dev["R"])
    _against_oracle(sb, out, oracle_t4, 1e-12)


@pytest.mark.parametrize("w12", [False, True])
def test_full_size_tensor_core_chain_matches_oracle(setup, oracle_t4, w12):
    sb, qn, lay, host, host_r, ctx, dev, chain = setup
    cm = sb.Context(0)
    cm.set_precision("tf32x3")
    dm = {n: sb.NewBlockSparseSorted(lay.dims[n], lay.n2[n], k, None, d, ctx=cm, block_dims=e)
          for n, (k, d, e) in host_r.items()}
    ch = qn.HeffChain(lay, cm, w12=w12, f32_intermediates=True)
    out = ch.apply(dm["psi"], dm["L"], dm["W1"], dm["W2"], dm["R"])
    cm.synchronize()
    worst = _against_oracle(sb, out, oracle_t4, 2e-5)
    print(f"chi={CHI} tf32x3 w12={w12}: worst block rel err vs oracle {worst:.2e}")
