"""C++ restatement of contract_shared! (block-sparse x block-sparse) on the
CPU, linked at run time to the OpenBLAS that numpy ships (scipy-openblas).

THIS PACKAGE IS TEST INFRASTRUCTURE: the CPU baseline of ``bench.py`` and a
second restatement the tests compare the numpy oracle with; the product path
never calls it.  ``build()`` compiles ``shared_bb.cpp`` in place with g++;
``contract_shared(...)`` runs one contraction on oracle ``BS`` tensors and
returns an oracle ``BS``; ``Tensor`` keeps operands resident in the C++ side
for repeated contractions (a timed chain)."""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "shared_bb.cpp")
LIB = os.path.join(HERE, "libshared_bb.so")

_lib = None
_blas = None


def build(force: bool = False) -> str:
    """g++ -O3 of shared_bb.cpp into libshared_bb.so beside it."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-o", LIB, SRC])
    return LIB


def openblas():
    """numpy's bundled OpenBLAS (the library numpy's own matmul calls)."""
    global _blas
    if _blas is None:
        d = os.path.join(os.path.dirname(np.__file__), os.pardir, "numpy.libs")
        cands = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so*")))
        if not cands:
            raise RuntimeError("numpy's bundled OpenBLAS (scipy-openblas) not found")
        _blas = C.CDLL(cands[0])
    return _blas


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError("oracle/cpu_ref/libshared_bb.so is not built (oracle.cpu_ref.build())")
        lib = C.CDLL(LIB)
        P, I64, VP = C.POINTER, C.c_int64, C.c_void_p
        lib.oref_set_dgemm.argtypes = [VP]
        lib.oref_last_error.restype = C.c_char_p
        lib.oref_new.argtypes = [C.c_int, P(I64), C.c_int, I64, P(I64), P(C.c_double), P(VP)]
        lib.oref_free.argtypes = [VP]
        lib.oref_info.argtypes = [VP, P(I64), P(I64)]
        lib.oref_export.argtypes = [VP, P(I64), P(C.c_double)]
        lib.oref_contract_shared.argtypes = [C.c_int, P(I64), C.c_int, P(I64), VP, P(I64), VP, P(I64), P(VP)]
        lib.oref_fuse_prefix.argtypes = [VP, C.c_int, C.c_int, P(VP)]
        lib.oref_contract_coo_prefix.argtypes = [C.c_int, P(I64), C.c_int, P(I64), C.c_int, P(I64), I64, P(I64),
                                                 P(C.c_double), P(I64), VP, P(I64), P(VP)]
        blas = openblas()
        fn = getattr(blas, "scipy_cblas_dgemm64_")
        lib.oref_set_dgemm(C.cast(fn, VP))
        _lib = lib
    return _lib


def set_threads(n: int) -> None:
    """OpenBLAS thread count for the dgemm calls."""
    openblas().scipy_openblas_set_num_threads64_(C.c_int(int(n)))


def _i64(xs):
    xs = [int(x) for x in xs]
    return (C.c_int64 * max(len(xs), 1))(*xs)


def _check(st: int) -> None:
    if st != 0:
        raise RuntimeError(load().oref_last_error().decode())


class Tensor:
    """A block-sparse tensor held by the C++ side (uniform reference layout)."""

    def __init__(self, dims: Sequence[int], n2: int, keys, data, _handle=None):
        lib = load()
        self.dims, self.n2 = tuple(int(d) for d in dims), int(n2)
        if _handle is not None:
            self._h = _handle
            return
        P = len(self.dims) - self.n2
        keys = [tuple(k) for k in keys]
        d = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(-1))
        h = C.c_void_p()
        _check(lib.oref_new(len(self.dims), _i64(self.dims), self.n2, len(keys), _i64([x for k in keys for x in k]),
                            d.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h)))
        self._h = h

    @staticmethod
    def from_bs(B) -> "Tensor":
        """From an oracle BS (blocks in key order)."""
        data = np.concatenate([B.block(i) for i in B.ids]) if B.keys else np.zeros(0)
        return Tensor(B.dims, B.n2, B.keys, data)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.oref_free(h)
            self._h = None

    def export(self):
        lib = load()
        n, blk = C.c_int64(), C.c_int64()
        _check(lib.oref_info(self._h, C.byref(n), C.byref(blk)))
        P = len(self.dims) - self.n2
        keys = (C.c_int64 * max(n.value * P, 1))()
        data = np.empty(n.value * blk.value)
        _check(lib.oref_export(self._h, keys, data.ctypes.data_as(C.POINTER(C.c_double))))
        return [tuple(keys[j * P + t] for t in range(P)) for j in range(n.value)], data

    def to_bs(self):
        from oracle import sparse_oracle as so
        keys, data = self.export()
        return so.BS(self.dims, self.n2, keys, list(range(1, len(keys) + 1)), data)


_LABEL_IDS: dict = {}


def _label_ids(labels):
    return [_LABEL_IDS.setdefault(l, len(_LABEL_IDS) + 1) for l in labels]


def contract(dimsC, n2C, labelsC, A: Tensor, labelsA, B: Tensor, labelsB) -> Tensor:
    """contract_shared! of two C++-side tensors into a new one."""
    lib = load()
    h = C.c_void_p()
    _check(lib.oref_contract_shared(len(dimsC), _i64(dimsC), int(n2C), _i64(_label_ids(labelsC)), A._h,
                                    _i64(_label_ids(labelsA)), B._h, _i64(_label_ids(labelsB)), C.byref(h)))
    return Tensor(dimsC, n2C, None, None, _handle=h)


def contract_shared(C0, labelsC, A, labelsA, B, labelsB):
    """Oracle-typed convenience: BS operands in, BS result out (C0 gives dims and n2)."""
    return contract(C0.dims, C0.n2, labelsC, Tensor.from_bs(A), labelsA, Tensor.from_bs(B), labelsB).to_bs()


def fuse_prefix(A: Tensor, ax1: int, ax2: int) -> Tensor:
    """fuse_two_axes! of two prefix axes (1-based)."""
    lib = load()
    h = C.c_void_p()
    _check(lib.oref_fuse_prefix(A._h, int(ax1), int(ax2), C.byref(h)))
    a1, a2 = min(ax1, ax2), max(ax1, ax2)
    dims = tuple(A.dims[a1 - 1] * A.dims[a2 - 1] if i == a1 else A.dims[i - 1]
                 for i in range(1, len(A.dims) + 1) if i != a2)
    return Tensor(dims, A.n2, None, None, _handle=h)


def contract_coo_prefix(dimsC, n2C, labelsC, A, labelsA, B: Tensor, labelsB) -> Tensor:
    """contract_prefix! with an oracle COO ``A`` and a C++-side ``B``."""
    lib = load()
    h = C.c_void_p()
    keys = [int(x) for k in A.keys for x in k]
    vals = np.ascontiguousarray(np.asarray(A.vals, dtype=np.float64))
    _check(lib.oref_contract_coo_prefix(len(dimsC), _i64(dimsC), int(n2C), _i64(_label_ids(labelsC)), len(A.dims),
                                        _i64(A.dims), len(A.vals), _i64(keys),
                                        vals.ctypes.data_as(C.POINTER(C.c_double)), _i64(_label_ids(labelsA)),
                                        B._h, _i64(_label_ids(labelsB)), C.byref(h)))
    return Tensor(dimsC, n2C, None, None, _handle=h)


def pxp_heff_runner(prob):
    """The PXP matvec (``sparsebackends_b200.pxp.HEFF_STEPS``) on the C++
    side for an ``oracle.pxp_oracle.OracleProblem``: returns ``apply(psi)``
    taking and returning C++ tensors, with L, R and psi resident."""
    from sparsebackends_b200 import pxp
    from oracle import sparse_oracle as so
    L, R, psi = Tensor.from_bs(prob.L), Tensor.from_bs(prob.R), Tensor.from_bs(prob.psi)

    def contract_any(lc, n2, A, la, B, lb):
        ext = dict(zip(la, A.dims))
        ext.update(zip(lb, B.dims))
        dims = tuple(ext[x] for x in lc)
        if isinstance(A, so.COO):
            return contract_coo_prefix(dims, n2, lc, A, la, B, lb)
        return contract(dims, n2, lc, A, la, B, lb)

    def apply(x):
        t = {"psi": x, "L": L, "R": R, "W1f": prob.Wf, "W2f": prob.Wf}
        return pxp.run_steps(pxp.HEFF_STEPS, t, dict(pxp.LABELS), contract_any, fuse_prefix)["T4"]

    return apply, psi
