"""The PXP centre problem on the oracle (numpy).

THIS MODULE IS TEST INFRASTRUCTURE, like ``oracle.sparse_oracle``: only
``tests/`` and the CPU-baseline leg of ``bench.py`` may import it.

It runs the step tables of ``sparsebackends_b200.pxp`` (environment updates
and the two-site H_eff matvec of the PXP chain, MPO in COO) with the oracle's
``contract`` (contract.jl:37-104), ``fuse_two_axes`` (blocksparse/
conversions.jl:228-314) and ``fuse_axes_coo`` (coo/conversions.jl:174-222):
the device path's label flow on the reference's algorithms.  The tables
themselves are checked against a dense einsum of the same Hamiltonian in
``tests/test_pxp_oracle.py``."""
from __future__ import annotations

from oracle import sparse_oracle as so
from sparsebackends_b200 import pxp


def o_contract(lc, n2, A, la, B, lb):
    """``contract!`` into a fresh block-sparse C with dims taken by label."""
    ext = dict(zip(la, so.dims_of(A)))
    ext.update(zip(lb, so.dims_of(B)))
    return so.contract(so.BS.empty(tuple(ext[x] for x in lc), n2), lc, A, la, B, lb)


def o_fuse(A, ax1, ax2):
    return so.fuse_axes_coo(A, ax1, ax2) if isinstance(A, so.COO) else so.fuse_two_axes(A, ax1, ax2)


def o_bs(dims, keys, data):
    return so.BS(dims, 2, list(keys), list(range(1, len(keys) + 1)), data)


def o_mpo():
    """(W, W with (s, wl) fused, W with (s, wr) fused) as oracle COO tensors."""
    keys, vals = pxp.mpo_entries()
    Wc = so.COO((pxp.D, pxp.D, pxp.W, pxp.W), list(keys), list(vals))
    Wf = so.fuse_axes_coo(so.coo_sort(so.coo_permutedims(Wc, [1, 4, 2, 3])), 3, 4)
    Wrf = so.fuse_axes_coo(so.coo_sort(so.coo_permutedims(Wc, [1, 3, 2, 4])), 3, 4)
    return Wc, Wf, Wrf


def o_run(steps, tensors):
    return pxp.run_steps(steps, tensors, dict(pxp.LABELS), o_contract, o_fuse)


class OracleProblem:
    """Oracle environments and operator of ``pxp.PxpProblem(n, chi, seed)``:
    the same random MPS, environments built from the boundaries by the same
    step tables."""

    def __init__(self, n, chi, seed):
        self.sites, self.psi_host, self.c = pxp.random_mps(n, chi, seed)
        self.Wc, self.Wf, self.Wrf = o_mpo()
        L = o_bs(*pxp.boundary_blocks(pxp.LEFT_CHANNEL))
        for k in range(1, self.c):
            A = o_bs(*pxp.site_blocks(self.sites[k - 1]))
            L = o_run(pxp.ENV_L_STEPS, {"L": L, "A": A, "Abar": A, "Wf": self.Wf})["out"]
        R = o_bs(*pxp.boundary_blocks(pxp.RIGHT_CHANNEL))
        for k in range(n, self.c + 1, -1):
            B = o_bs(*pxp.site_blocks(self.sites[k - 1]))
            R = o_run(pxp.ENV_R_STEPS, {"R": R, "A": B, "Abar": B, "Wrf": self.Wrf})["out"]
        self.L, self.R = L, R
        self.psi = o_bs(*pxp.psi_blocks(self.psi_host))

    def apply(self, psi):
        """H_eff . psi (the table HEFF_STEPS)."""
        return o_run(pxp.HEFF_STEPS, {"psi": psi, "L": self.L, "R": self.R, "W1f": self.Wf, "W2f": self.Wf})["T4"]

    def apply_aliased(self, psi_d):
        """H_eff . psi with W aliased and dense psi (l, s1, s2, r) and
        environments (the table ALIASED_HEFF_STEPS); returns the dense result."""
        dims, tm, keys, aids, sc = pxp.mpo_aliased()
        Wa = so.Aliased(dims, 2, tm, 3, list(keys), list(aids), list(sc))
        ops = {"W1a": Wa, "W2a": Wa, "psi_d": psi_d,
               "Ld": pxp.env_dense(self.L.keys, self.L.blocks_by_key(), self.L.dims, right=False),
               "Rd": pxp.env_dense(self.R.keys, self.R.blocks_by_key(), self.R.dims, right=True)}

        def contract(lc, n2, A, la, B, lb):
            ext = dict(zip(la, so.dims_of(A)))
            ext.update(zip(lb, so.dims_of(B)))
            return so.contract(so.Aliased.empty(tuple(ext[x] for x in lc), n2), lc, A, la, B, lb)

        X4 = pxp.run_steps(pxp.ALIASED_HEFF_STEPS, ops, dict(pxp.ALIASED_LABELS), contract, None)["X4"]
        return X4

    def apply_mpo(self, A):
        """MPO x MPS on one oracle site tensor (contract_prefix!)."""
        dims = (pxp.D, pxp.W, pxp.W, 1, 1) + tuple(A.dims[3:])
        return so.contract(so.BS.empty(dims, 2), ["sp", "wl", "wr", "ql", "qr", "l", "r"], self.Wc,
                           ["sp", "s", "wl", "wr"], A, ["ql", "s", "qr", "l", "r"])
