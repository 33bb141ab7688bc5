"""Contractions on which the two merge-join orders of contract_shared! are
compared: the reference's known-answer cases and the H_eff / environment
contractions of two workloads, on seeded operands that fill every
charge-allowed block.

* centre problem: Heisenberg N = 16, chi = 64 (links ``dmrg.profile_link``),
  the XXZ MPO's own blocks (w = 5), the two-site chain at the centre bond (both
  associations), ``make_L`` at site 8, ``make_R`` at site 9, and the first
  update ``make_L`` from the boundary environment at site 1;
* J1-J2 6x6-sized problem: U(1) sectors 2Sz = -10..10 of chi = 64 (Gaussian
  profile, odd charges on the link past one site), MPO link of 38 channels
  on every allowed block, the same contractions.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

from oracle import sparse_oracle as so


def _bs(dims, n2, blocks: Dict[Tuple[int, ...], np.ndarray]):
    keys = sorted(blocks, key=lambda k: k[::-1])
    data = np.concatenate([blocks[k].reshape(-1, order="F") for k in keys]) if keys else np.zeros(0)
    return so.BS(tuple(dims), n2, keys, list(range(1, len(keys) + 1)), data)


def _random(lay, name, rng):
    from sparsebackends_b200 import qn
    keys, data = qn.random_block_tensor(lay, name, rng, 1.0)
    return so.BS(lay.dims[name], lay.n2[name], keys, list(range(1, len(keys) + 1)), data)


def _xxz_mpo(lay):
    from sparsebackends_b200 import dmrg
    D = dmrg.MPO_LINK.D
    blocks = {}
    for k, m in dmrg.mpo_blocks(1.0).items():
        pad = np.zeros((D, D))
        pad[: m.shape[0], : m.shape[1]] = m
        blocks[k] = pad
    return _bs(lay.dims["W1"], 2, blocks)


def _chain_cases(tag, lay, t):
    from sparsebackends_b200 import qn
    lab = lay.labels
    out = []
    for steps, assoc in ((qn.HeffChain.STEPS, "chain"), (qn.HeffChain.STEPS_W12, "chain_w12")):
        tt = dict(t)
        for c, a, b in steps:
            out.append((f"{tag}:{assoc}:{c}={a}*{b}", so.BS.empty(lay.dims[c], lay.n2[c]), lab[c],
                        tt[a], lab[a], tt[b], lab[b]))
            tt[c] = so.contract(so.BS.empty(lay.dims[c], lay.n2[c]), lab[c], tt[a], lab[a], tt[b], lab[b])
    return out


def _env_cases(tag, steps, E, A, W, names):
    """The three contractions of one environment update (results of the
    sorted-order merge feed the next step)."""
    out = []
    left = E
    for (lc, n2c, la, lb), right, nm in zip(steps, (A, W, A), names):
        dims = {}
        for l, d in zip(la, left.dims):
            dims[l] = d
        for l, d in zip(lb, right.dims):
            dims[l] = d
        C0 = so.BS.empty(tuple(dims[l] for l in lc), n2c)
        out.append((f"{tag}:{nm}", C0, lc, left, la, right, lb))
        left = so.contract(so.BS.empty(C0.dims, n2c), lc, left, la, right, lb)
    return out


def centre_problem_cases():
    from sparsebackends_b200 import dmrg, qn
    rng = np.random.Generator(np.random.PCG64(41))
    links = [dmrg.profile_link(16, b) for b in range(17)]
    lay = qn.HeffLayout(links[7], links[9], dmrg.MPO_LINK)
    W = _xxz_mpo(lay)
    t = {"psi": _random(lay, "psi", rng), "L": _random(lay, "L", rng), "W1": W, "W2": W,
         "R": _random(lay, "R", rng)}
    out = _chain_cases("n16", lay, t)
    la = qn.HeffLayout(links[7], links[8], dmrg.MPO_LINK)  # site 8: A from link 7 to link 8, L on link 7
    out += _env_cases("n16:make_L(site 8)", qn.MAKE_L_STEPS, _random(la, "L", rng), _random(la, "A", rng), W,
                      ("E1=L*A", "E2=E1*W", "L'=E2*A"))
    lr = qn.HeffLayout(links[8], links[9], dmrg.MPO_LINK)  # site 9: B from link 8 to link 9, R on link 9
    out += _env_cases("n16:make_R(site 9)", qn.MAKE_R_STEPS, _random(lr, "R", rng), _random(lr, "A", rng), W,
                      ("F1=R*B", "F2=F1*W", "R'=F2*B"))
    # the first update from the boundary: L0 holds only the "identity before" channel
    l0 = qn.HeffLayout(links[0], links[1], dmrg.MPO_LINK)
    q0 = dmrg.MPO_LINK.index(0) + 1
    blk = np.zeros((1, dmrg.MPO_LINK.D, 1))
    blk[0, dmrg.CHANNEL[1][1] - 1, 0] = 1.0
    L0 = _bs(l0.dims["L"], 3, {(1, q0, 1): blk})
    out += _env_cases("n16:make_L(site 1, boundary)", qn.MAKE_L_STEPS, L0, _random(l0, "A", rng), W,
                      ("E1=L0*A", "E2=E1*W", "L'=E2*A"))
    return out


def j1j2_sized_cases(chi: int = 64):
    from sparsebackends_b200 import qn
    rng = np.random.Generator(np.random.PCG64(43))
    even = qn.gaussian_sectors(chi, list(range(-10, 11, 2)), width=2.0)
    odd = qn.gaussian_sectors(chi, list(range(-9, 10, 2)), width=2.0)
    mpo = qn.mpo_link({-2: 12, 0: 14, 2: 12})
    lay = qn.HeffLayout(even, even, mpo)
    t = {n: _random(lay, n, rng) for n in ("psi", "L", "W1", "W2", "R")}
    out = _chain_cases("j1j2", lay, t)
    la = qn.HeffLayout(even, odd, mpo)
    W = _random(la, "W1", rng)
    out += _env_cases("j1j2:make_L", qn.MAKE_L_STEPS, _random(la, "L", rng), _random(la, "A", rng), W,
                      ("E1=L*A", "E2=E1*W", "L'=E2*A"))
    lr = qn.HeffLayout(odd, even, mpo)
    out += _env_cases("j1j2:make_R", qn.MAKE_R_STEPS, _random(lr, "R", rng), _random(lr, "A", rng), W,
                      ("F1=R*B", "F2=F1*W", "R'=F2*B"))
    return out


def compare_join_orders(C0, lc, A, la, B, lb) -> dict:
    """Both merge orders on one contraction: key lists, missing keys and the
    largest relative block difference of the reference order's result."""
    got = so.contract(so.BS.empty(C0.dims, C0.n2), lc, A, la, B, lb)
    with so.join_order("reference"):
        ref = so.contract(so.BS.empty(C0.dims, C0.n2), lc, A, la, B, lb)
    gb, rb = got.blocks_by_key(), ref.blocks_by_key()
    worst = 0.0
    for k, v in gb.items():
        w = rb.get(k)
        d = np.linalg.norm(v - (w if w is not None else 0.0))
        worst = max(worst, float(d / max(np.linalg.norm(v), 1e-300)))
    return {"same_keys": got.keys == ref.keys, "missing": len(set(got.keys) - set(ref.keys)),
            "extra": len(set(ref.keys) - set(got.keys)), "nkeys": len(got.keys),
            "max_rel_diff": worst, "njoin": _njoin(lc, la, A.P, lb, B.P)}


def _njoin(lc, la, PA, lb, PB) -> int:
    return sum(1 for l in la[:PA] if l in lb[:PB] and l not in lc)
