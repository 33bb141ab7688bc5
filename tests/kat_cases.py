"""Known-answer cases restated from the reference's own tests.

Each case carries the reference test it comes from (paths relative to the
``SparseBackends`` package).  Inputs are the hand-placed nonzeros of those
tests (1-based Julia indices converted to 0-based numpy indices); expected
outputs are the tests' dense references (one GEMM over permuted operands),
converted back with ``blocksparse_from_dense(...; atol=0, rtol=0)``.

The same cases drive the oracle KAT tests (CPU) and the CUDA parity tests
(GPU), so both are pinned to the reference's fixtures.
"""
from __future__ import annotations

import itertools
import string
from dataclasses import dataclass
from typing import Any, List, Optional

import numpy as np


def dense_contract(A, la, B, lb, lc):
    """Dense reference: sum over labels shared by A and B, output in lc order."""
    letters = {}
    for l in list(la) + list(lb) + list(lc):
        if l not in letters:
            letters[l] = string.ascii_letters[len(letters)]
    spec = "".join(letters[l] for l in la) + "," + "".join(letters[l] for l in lb) + "->" + "".join(letters[l] for l in lc)
    return np.einsum(spec, A, B, optimize=False)


def permute_from_canon(X, canon, target):
    pos = {l: i for i, l in enumerate(canon)}
    return np.ascontiguousarray(np.transpose(X, [pos[l] for l in target]))


@dataclass
class Case:
    name: str
    source: str
    kind_A: str  # "bs", "coo", "dense"
    kind_B: str
    kind_C: str  # "bs", "coo"
    A: np.ndarray
    labelsA: List[str]
    n2A: int
    B: np.ndarray
    labelsB: List[str]
    n2B: int
    labelsC: List[str]
    n2C: int
    expect_error: bool = False

    @property
    def C_dense(self):
        return dense_contract(self.A, self.labelsA, self.B, self.labelsB, self.labelsC)

    @property
    def dimsC(self):
        d = {}
        for l, s in zip(self.labelsA, self.A.shape):
            d[l] = s
        for l, s in zip(self.labelsB, self.B.shape):
            d[l] = s
        return tuple(d[l] for l in self.labelsC)


def bs_dense_cases() -> List[Case]:
    """test/tensoralgebra/bs_dense.jl:102-181 (r in A prefix, B dense)."""
    I, J, R, XA, XB = 3, 2, 4, 2, 3
    A_canon = np.zeros((I, R, XA))
    B_canon = np.zeros((J, R, XB))
    A_canon[0, 0, 0] = 2.0
    A_canon[1, 0, 1] = -1.0
    A_canon[2, 2, 0] = 0.5
    A_canon[0, 3, 1] = 1.5
    B_canon[0, 0, 1] = 7.0
    B_canon[1, 0, 0] = -2.0
    B_canon[1, 2, 2] = 1.0
    B_canon[0, 3, 0] = 0.25
    out = []
    for la, lb, lc in itertools.product(
        [["i", "r", "xa"], ["r", "i", "xa"]],
        [["j", "r", "xb"], ["r", "j", "xb"], ["j", "xb", "r"]],
        [["i", "xa", "j", "xb"], ["i", "j", "xb", "xa"]],
    ):
        A = permute_from_canon(A_canon, ["i", "r", "xa"], la)
        B = permute_from_canon(B_canon, ["j", "r", "xb"], lb)
        out.append(Case(f"bs_dense[{la}|{lb}|{lc}]", "test/tensoralgebra/bs_dense.jl:102-181",
                        "bs", "dense", "bs", A, la, 1, B, lb, 0, lc, 3))
    return out


def bs_bs_prefix_cases() -> List[Case]:
    """test/tensoralgebra/bs_bs.jl:210-299 (r in both prefixes)."""
    I, J, R, XA, XB = 3, 2, 4, 2, 3
    A_canon = np.zeros((I, R, XA))
    B_canon = np.zeros((J, R, XB))
    A_canon[0, 0, 0] = 2.0
    A_canon[1, 0, 1] = -1.0
    A_canon[2, 2, 0] = 0.5
    A_canon[0, 3, 1] = 1.5
    B_canon[0, 0, 1] = 7.0
    B_canon[1, 0, 0] = -2.0
    B_canon[1, 2, 2] = 1.0
    B_canon[0, 3, 0] = 0.25
    out = []
    for la, lb, lc in itertools.product(
        [["i", "r", "xa"], ["r", "i", "xa"]],
        [["j", "r", "xb"], ["r", "j", "xb"]],
        [["i", "j", "xa", "xb"], ["i", "j", "xb", "xa"], ["j", "i", "xa", "xb"], ["j", "i", "xb", "xa"]],
    ):
        A = permute_from_canon(A_canon, ["i", "r", "xa"], la)
        B = permute_from_canon(B_canon, ["j", "r", "xb"], lb)
        out.append(Case(f"bs_bs_prefix[{la}|{lb}|{lc}]", "test/tensoralgebra/bs_bs.jl:210-299",
                        "bs", "bs", "bs", A, la, 1, B, lb, 1, lc, 2))
    return out


def bs_bs_dense_cases() -> List[Case]:
    """test/tensoralgebra/bs_bs.jl:301-387 (r in both dense tails)."""
    PA, PB, A1, B1, R = 2, 3, 4, 5, 3
    A_can = np.zeros((PA, A1, R))
    B_can = np.zeros((PB, B1, R))
    A_can[0, 0, 0] = 2.0
    A_can[1, 2, 1] = -1.0
    A_can[0, 3, 2] = 0.5
    B_can[0, 1, 0] = 7.0
    B_can[2, 4, 1] = -2.0
    B_can[1, 0, 2] = 1.0
    out = []
    for la, lb, lc in itertools.product(
        [["pa", "a1", "r"], ["pa", "r", "a1"]],
        [["pb", "b1", "r"], ["pb", "r", "b1"]],
        [["pa", "pb", "a1", "b1"], ["pa", "pb", "b1", "a1"], ["pb", "pa", "a1", "b1"], ["pb", "pa", "b1", "a1"]],
    ):
        A = permute_from_canon(A_can, ["pa", "a1", "r"], la)
        B = permute_from_canon(B_can, ["pb", "b1", "r"], lb)
        out.append(Case(f"bs_bs_dense[{la}|{lb}|{lc}]", "test/tensoralgebra/bs_bs.jl:301-387",
                        "bs", "bs", "bs", A, la, 2, B, lb, 2, lc, 2))
    return out


def bs_bs_multi_cases() -> List[Case]:
    """test/tensoralgebra/bs_bs_multi_labels.jl:172-270 (+ the :272-301 error case)."""
    I, J, R1, R2, XA1, XA2, K1, K2, XB = 2, 3, 2, 2, 2, 2, 2, 2, 2
    la_can = ["i", "r1", "r2", "xa1", "xa2", "k1", "k2"]
    lb_can = ["j", "r1", "r2", "k1", "k2", "xb"]
    A_canon = np.zeros((I, R1, R2, XA1, XA2, K1, K2))
    B_canon = np.zeros((J, R1, R2, K1, K2, XB))
    A_canon[0, 0, 0, 0, 1, 0, 1] = 2.0
    A_canon[0, 1, 0, 1, 0, 1, 0] = -1.0
    A_canon[1, 0, 1, 0, 0, 1, 1] = 0.5
    A_canon[1, 1, 1, 1, 1, 0, 0] = 1.5
    B_canon[0, 0, 0, 0, 1, 1] = 7.0
    B_canon[0, 1, 0, 1, 0, 0] = -2.0
    B_canon[2, 0, 1, 1, 1, 1] = 1.0
    B_canon[1, 1, 1, 0, 0, 0] = 0.25
    PA, PB = 3, 3
    shared_pref, shared_den = ["r1", "r2"], ["k1", "k2"]

    def valid(l, P):
        return all(l.index(x) < P for x in shared_pref) and all(l.index(x) >= P for x in shared_den)

    las = [l for l in [la_can, ["r1", "i", "r2", "xa2", "xa1", "k2", "k1"], ["r2", "r1", "i", "k1", "xa1", "xa2", "k2"]]
           if valid(l, PA)]
    lbs = [l for l in [lb_can, ["r2", "j", "r1", "k2", "xb", "k1"], ["r1", "r2", "j", "xb", "k1", "k2"]]
           if valid(l, PB)]
    lcs = [["i", "j", "xa1", "xa2", "xb"], ["i", "j", "xa2", "xa1", "xb"], ["j", "i", "xa2", "xa1", "xb"],
           ["i", "j", "xb", "xa1", "xa2"], ["j", "i", "xb", "xa2", "xa1"]]
    out = []
    for la, lb, lc in itertools.product(las, lbs, lcs):
        A = permute_from_canon(A_canon, la_can, la)
        B = permute_from_canon(B_canon, lb_can, lb)
        out.append(Case(f"bs_bs_multi[{la}|{lb}|{lc}]", "test/tensoralgebra/bs_bs_multi_labels.jl:172-270",
                        "bs", "bs", "bs", A, la, 4, B, lb, 3, lc, 3))
    # interleaved C dense order must raise
    A_d = np.zeros((2,) * 7)
    B_d = np.zeros((2,) * 6)
    A_d[(0,) * 7] = 1.0
    B_d[(0,) * 6] = 2.0
    out.append(Case("bs_bs_multi[interleaved]", "test/tensoralgebra/bs_bs_multi_labels.jl:272-301",
                    "bs", "bs", "bs", A_d, la_can, 4, B_d, lb_can, 3,
                    ["i", "j", "xa1", "xb", "xa2"], 3, expect_error=True))
    return out


def coo_bs_cases() -> List[Case]:
    """test/tensoralgebra/coo_bs.jl:21-250 (five configurations)."""
    out = []
    A = np.zeros((3, 4)); A[0, 0] = 2.0; A[2, 1] = -1.0; A[1, 3] = 0.5
    B = np.zeros((4, 2, 3)); B[0, 0, 1] = 7.0; B[1, 1, 0] = -2.0; B[3, 0, 2] = 1.0
    out.append(Case("coo_bs[i,r x r,j,k]", "test/tensoralgebra/coo_bs.jl:22-60",
                    "coo", "bs", "bs", A, ["i", "r"], 0, B, ["r", "j", "k"], 2, ["i", "j", "k"], 2))
    A = np.zeros((4, 3)); A[0, 0] = 2.0; A[1, 2] = -1.0; A[3, 1] = 0.5
    B = np.zeros((4, 2, 2)); B[0, 0, 1] = 7.0; B[1, 1, 0] = -2.0; B[3, 0, 0] = 1.0
    out.append(Case("coo_bs[r,i x r,j,k]", "test/tensoralgebra/coo_bs.jl:62-107",
                    "coo", "bs", "bs", A, ["r", "i"], 0, B, ["r", "j", "k"], 2, ["i", "j", "k"], 2))
    A = np.zeros((2, 3, 4)); A[0, 0, 0] = 2.0; A[1, 2, 1] = -1.0; A[0, 1, 3] = 3.5
    B = np.zeros((4, 2, 2)); B[0, 0, 1] = 7.0; B[1, 1, 0] = -2.0; B[3, 0, 0] = 1.0
    out.append(Case("coo_bs[i,p,r x r,j,k]", "test/tensoralgebra/coo_bs.jl:109-148",
                    "coo", "bs", "bs", A, ["i", "p", "r"], 0, B, ["r", "j", "k"], 2, ["i", "p", "j", "k"], 2))
    A = np.zeros((3, 4)); A[0, 0] = 2.0; A[2, 1] = -1.0; A[1, 3] = 0.5
    B = np.zeros((2, 3, 4)); B[0, 0, 0] = 7.0; B[1, 1, 1] = -2.0; B[0, 2, 3] = 1.0
    out.append(Case("coo_bs[i,r x j,x,r]", "test/tensoralgebra/coo_bs.jl:150-199",
                    "coo", "bs", "bs", A, ["i", "r"], 0, B, ["j", "x", "r"], 2, ["i", "j", "x"], 1))
    A = np.zeros((2, 3)); A[0, 0] = 1.0; A[1, 2] = -2.0
    B = np.zeros((3, 3, 2)); B[0, 0, 0] = 4.0; B[1, 1, 1] = 5.0; B[2, 2, 0] = -1.0
    out.append(Case("coo_bs[i,r x j,r,x]", "test/tensoralgebra/coo_bs.jl:201-249",
                    "coo", "bs", "bs", A, ["i", "r"], 0, B, ["j", "r", "x"], 2, ["i", "j", "x"], 1))
    return out


def coo_dense_cases() -> List[Case]:
    """test/tensoralgebra/coo_dense.jl:72-161 (Config1, Config2)."""
    out = []
    A_ir = np.zeros((3, 4)); A_ir[0, 0] = 2.0; A_ir[2, 1] = -1.0; A_ir[1, 3] = 0.5
    B_xr = np.zeros((5, 4)); B_xr[1, 0] = 7.0; B_xr[4, 1] = -2.0; B_xr[0, 3] = 1.0
    for la, lb in itertools.product([["i", "r"], ["r", "i"]], [["x", "r"], ["r", "x"]]):
        A = permute_from_canon(A_ir, ["i", "r"], la)
        B = permute_from_canon(B_xr, ["x", "r"], lb)
        out.append(Case(f"coo_dense1[{la}|{lb}]", "test/tensoralgebra/coo_dense.jl:72-107",
                        "coo", "dense", "bs", A, la, 0, B, lb, 0, ["i", "x"], 1))
    A_pir = np.zeros((2, 3, 4)); A_pir[0, 0, 0] = 2.0; A_pir[1, 2, 1] = -1.0; A_pir[0, 1, 3] = 0.5
    B_yxr = np.zeros((3, 2, 4)); B_yxr[0, 1, 0] = 7.0; B_yxr[2, 0, 1] = -2.0; B_yxr[1, 1, 3] = 1.0
    for la, lb, lc in itertools.product(
        [["p", "i", "r"], ["i", "p", "r"], ["r", "p", "i"]],
        [["y", "x", "r"], ["x", "y", "r"], ["r", "y", "x"]],
        [["p", "i", "y", "x"], ["i", "p", "y", "x"], ["p", "i", "x", "y"], ["i", "p", "x", "y"]],
    ):
        A = permute_from_canon(A_pir, ["p", "i", "r"], la)
        B = permute_from_canon(B_yxr, ["y", "x", "r"], lb)
        out.append(Case(f"coo_dense2[{la}|{lb}|{lc}]", "test/tensoralgebra/coo_dense.jl:109-161",
                        "coo", "dense", "bs", A, la, 0, B, lb, 0, lc, 2))
    return out


def coo_coo_cases() -> List[Case]:
    """test/tensoralgebra/coo.jl:9-76."""
    A = np.zeros((3, 4)); A[0, 0] = 1.0; A[2, 1] = -2.0; A[1, 3] = 3.0
    B = np.zeros((4, 2)); B[0, 1] = 5.0; B[1, 0] = -1.0; B[3, 1] = 2.0
    c1 = Case("coo_coo[2d]", "test/tensoralgebra/coo.jl:9-36", "coo", "coo", "coo",
              A, ["i", "r"], 0, B, ["r", "j"], 0, ["i", "j"], 0)
    A = np.zeros((2, 3, 4)); A[0, 0, 0] = 2.0; A[1, 2, 1] = -1.0; A[0, 1, 3] = 3.5
    B = np.zeros((4, 2, 2)); B[0, 0, 1] = 7.0; B[1, 1, 0] = -2.0; B[3, 0, 0] = 1.0
    c2 = Case("coo_coo[3d]", "test/tensoralgebra/coo.jl:38-76", "coo", "coo", "coo",
              A, ["a", "b", "r"], 0, B, ["r", "c", "d"], 0, ["a", "b", "c", "d"], 0)
    return [c1, c2]


def all_cases() -> List[Case]:
    return (bs_dense_cases() + bs_bs_prefix_cases() + bs_bs_dense_cases() + bs_bs_multi_cases()
            + coo_bs_cases() + coo_dense_cases() + coo_coo_cases())
