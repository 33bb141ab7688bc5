"""B200-native block-sparse tensor contraction (drop-in for SparseBackends' contract!).

Python mirror of the reference's Julia API (``SparseBackends.jl`` exports and
``tensoralgebra/contract.jl``), backed by the CUDA library ``libsparseb.so``
through its C ABI.  Every tensor payload lives in device memory and every
floating-point result is computed by CUDA kernels on the GPU; there is no CPU
fallback — without a CUDA device, operations raise :class:`SparseBackendsError`.

Names follow the reference:

=============================  ==========================================================
``NewBlockSparseSorted``       ``src/blocksparse/storage.jl:3-9``
``COOTensor``                  ``src/coo/storage.jl:1-6``
``AliasedBlockSparse``         ``src/aliased/storage.jl:46-54``
``DenseTensor``                the ``Array`` operands of ``contract!``
``contract_``                  ``contract!(C, labelsC, A, labelsA, B, labelsB)`` (contract.jl:37-104)
``contract_bs_bs_to_dense``    ``contract_bs_bs_to_dense!`` (contract_bs_bs.jl:736-754)
``blocksparse_from_dense``     ``src/blocksparse/conversions.jl:21-75``
``coo_from_dense``             ``src/coo/conversions.jl:13-26``
``to_dense`` / ``to_blocksparse``  conversions of all three formats
``permutedims`` / ``sort_``    ``permutedims`` / ``sort!`` of the storage types
``output_inds``                output index order of ``src/tensor_wrappers.jl:477-526``
=============================  ==========================================================

Labels are ``(id, plev)`` integer pairs as in the reference (``Label =
NTuple{2,UInt64}``); any other hashable label is mapped to a stable 64-bit id
with prime level 0.
"""
from __future__ import annotations

import ctypes as C
import hashlib
from typing import Any, Iterable, List, Optional, Sequence, Tuple, Callable

import numpy as np

from . import _lib

__all__ = [
    "SparseBackendsError", "Context", "Graph", "default_context", "DenseTensor", "NewBlockSparseSorted", "COOTensor",
    "AliasedBlockSparse", "contract_", "contract_bs_bs_to_dense", "blocksparse_from_dense", "coo_from_dense",
    "to_dense", "to_blocksparse", "permutedims", "sort_", "compression_ratio", "output_inds", "label_key",
    "to_uniform", "to_ragged", "crop_padding", "norm", "dot", "inner", "copy", "similar", "scale_", "fill_", "map_", "axpy_",
    "axpby_", "add", "MAP_AXPY", "MAP_AXPBY", "MAP_COPY", "MAP_MUL", "blocksparse_left_qr", "blocksparse_svd",
    "fuse_axes",
]


class SparseBackendsError(RuntimeError):
    """A failed library call; ``status`` is the sb_status name (e.g. ``SB_ERR_LABEL``)."""

    def __init__(self, status: int, message: str):
        self.code = status
        self.status = _lib.STATUS.get(status, str(status))
        super().__init__(f"{self.status}: {message}")


def _check(ctx: Optional["Context"], st: int) -> None:
    if st != 0:
        lib = _lib.load()
        msg = lib.sb_last_error(ctx._h if ctx is not None else None)
        raise SparseBackendsError(st, (msg or b"").decode())


def label_key(lab: Any) -> Tuple[int, int]:
    """Map a label to the reference's ``(id, plev)`` pair of UInt64."""
    if isinstance(lab, tuple) and len(lab) == 2 and all(isinstance(x, (int, np.integer)) for x in lab):
        return int(lab[0]) & 0xFFFFFFFFFFFFFFFF, int(lab[1]) & 0xFFFFFFFFFFFFFFFF
    h = hashlib.blake2b(repr(lab).encode(), digest_size=8).digest()
    return int.from_bytes(h, "little"), 0


# Packed label arrays of label lists made of strings, by the tuple of strings
# (strings compare and hash by value, so a hit is exact).  The C side copies
# the labels, so one array serves every call; the cache is bounded.
_LABELS_CACHE: dict = {}
_LABELS_CACHE_MAX = 4096


def _labels(labels: Sequence[Any]):
    key = tuple(labels)
    strs = all(type(l) is str for l in key)
    if strs:
        hit = _LABELS_CACHE.get(key)
        if hit is not None:
            return hit
    flat = []
    for l in key:
        flat.extend(label_key(l))
    out = ((C.c_uint64 * max(len(flat), 1))(*flat), len(key))
    if strs and len(_LABELS_CACHE) < _LABELS_CACHE_MAX:
        _LABELS_CACHE[key] = out
    return out


def _i64(xs) -> "C.Array":
    xs = [int(x) for x in xs]
    return (C.c_int64 * max(len(xs), 1))(*xs)


def _f64ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """One CUDA device + stream (``sb_ctx``).  Tensors keep their context alive."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self._lib = _lib.load()
        h = C.c_void_p()
        _check(None, self._lib.sb_ctx_create(int(device), 0, C.byref(h)))
        self._h = h
        self.device = device
        if stream is not None:
            _check(self, self._lib.sb_ctx_set_stream(self._h, C.c_void_p(stream)))

    def synchronize(self) -> None:
        _check(self, self._lib.sb_ctx_synchronize(self._h))

    @property
    def stream(self) -> int:
        return self._lib.sb_ctx_get_stream(self._h) or 0

    def set_stream(self, stream: int) -> None:
        _check(self, self._lib.sb_ctx_set_stream(self._h, C.c_void_p(stream)))

    @property
    def launch_count(self) -> int:
        return int(self._lib.sb_ctx_launch_count(self._h))

    PROFILE_KINDS = {"gemm": 0, "permute": 1, "outer": 2, "axpy": 3, "other": 4, "vector": 5, "gemm_thin": 6,
                     "gemm_tc": 7, "tc_pack": 8}

    PRECISIONS = {"f64": 0, "tf32x3": 1, "tf32": 2}

    @property
    def precision(self) -> str:
        """Arithmetic of the tiled block GEMMs: "f64" (default, the drop-in),
        "tf32x3" (tcgen05, operands split into TF32 hi + lo) or "tf32"."""
        v = int(self._lib.sb_ctx_get_precision(self._h))
        return {b: a for a, b in self.PRECISIONS.items()}[v]

    def set_precision(self, precision: str) -> None:
        _check(self, self._lib.sb_ctx_set_precision(self._h, self.PRECISIONS[precision]))

    def set_profiling(self, enable: bool) -> None:
        """Time every kernel launch with CUDA events on the context stream."""
        _check(self, self._lib.sb_ctx_set_profiling(self._h, int(bool(enable))))

    def profile(self, kind: str = "gemm") -> dict:
        """Launch count, total ms, algorithmic FLOPs and bytes of one kernel class."""
        n, ms, fl, by = C.c_int64(), C.c_double(), C.c_double(), C.c_double()
        _check(self, self._lib.sb_ctx_profile_summary(self._h, self.PROFILE_KINDS[kind], C.byref(n), C.byref(ms),
                                                      C.byref(fl), C.byref(by)))
        return dict(launches=n.value, ms=ms.value, flops=fl.value, bytes=by.value)

    def capture(self, fn: Callable[[], Any], keep: Sequence[Any] = ()) -> "Graph":
        """Capture the library calls that ``fn()`` makes on this context into a
        CUDA graph (sb_ctx_capture_begin/end).  Run ``fn`` once eagerly before,
        so that its outputs already have their storage.  ``keep``: tensors the
        graph reads or writes; the Graph holds them so they outlive it."""
        _check(self, self._lib.sb_ctx_capture_begin(self._h))
        try:
            fn()
        finally:
            g = C.c_void_p()
            st = self._lib.sb_ctx_capture_end(self._h, C.byref(g))
        _check(self, st)
        return Graph(self, g, keep)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(self, "_lib", None)
        if h is not None and h.value and lib is not None:
            lib.sb_ctx_destroy(h)  # deferred by the library while tensors are alive
            self._h = None


class Graph:
    """A captured sequence of library calls, replayed on its context's stream.
    Each replay recomputes the captured outputs from the current device values
    of the captured inputs (same tensors, same block structure)."""

    def __init__(self, ctx: Context, handle: C.c_void_p, keep: Sequence[Any] = ()):
        self.ctx = ctx
        self._h = handle
        self._keep = list(keep)

    def launch(self) -> None:
        _check(self.ctx, self.ctx._lib.sb_graph_launch(self.ctx._h, self._h))

    def hold(self, *tensors: Any) -> None:
        """Keep tensors alive as long as the graph: outputs that the captured
        calls created (their storage was allocated at capture, and every
        replay writes it)."""
        self._keep.extend(tensors)

    def __del__(self):
        h = getattr(self, "_h", None)
        ctx = getattr(self, "ctx", None)
        if h is not None and h.value and ctx is not None and getattr(ctx, "_lib", None) is not None:
            ctx._lib.sb_graph_free(h)
            self._h = None


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class _Tensor:
    kind = -1

    def __init__(self, ctx: Context, handle: C.c_void_p):
        self.ctx = ctx
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        ctx = getattr(self, "ctx", None)
        if h is not None and h.value and ctx is not None and getattr(ctx, "_lib", None) is not None:
            ctx._lib.sb_tensor_free(h)
            self._h = None

    def _info(self):
        lib = self.ctx._lib
        kind, nd, n2, dirty = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        nkeys, blk, ntm = C.c_int64(), C.c_int64(), C.c_int64()
        _check(self.ctx, lib.sb_tensor_info(self._h, C.byref(kind), C.byref(nd), None, C.byref(n2), C.byref(nkeys),
                                            C.byref(blk), C.byref(ntm), C.byref(dirty)))
        dims = (C.c_int64 * max(nd.value, 1))()
        _check(self.ctx, lib.sb_tensor_info(self._h, None, None, dims, None, None, None, None, None))
        return dict(kind=kind.value, dims=tuple(dims[i] for i in range(nd.value)), n2=n2.value, nkeys=nkeys.value,
                    blksize=blk.value, n_templates=ntm.value, dirty=bool(dirty.value))

    @property
    def dims(self) -> Tuple[int, ...]:
        # a tensor's dims never change after creation (contract! and the
        # vector-space updates rewrite keys and payload only)
        d = self.__dict__.get("_dims")
        if d is None:
            d = self._dims = self._info()["dims"]
        return d

    def size(self) -> Tuple[int, ...]:
        return self.dims

    @property
    def ndim(self) -> int:
        return len(self.dims)

    def device_ptr(self) -> Tuple[int, int]:
        p, n = C.c_void_p(), C.c_int64()
        _check(self.ctx, self.ctx._lib.sb_tensor_device_data(self._h, C.byref(p), C.byref(n)))
        return p.value or 0, n.value

    # vector-space hooks (src/tensor_wrappers.jl:793-923): alpha*x, -x, x/alpha, x+y, x-y
    def __rmul__(self, alpha: float) -> "_Tensor":
        out = copy(self)
        return scale_(out, alpha)

    def __mul__(self, alpha: float) -> "_Tensor":
        return self.__rmul__(alpha)

    def __neg__(self) -> "_Tensor":
        return (-1.0) * self

    def __truediv__(self, alpha: float) -> "_Tensor":
        return (1.0 / alpha) * self

    def __add__(self, other: "_Tensor") -> "_Tensor":
        return add(self, other)

    def __sub__(self, other: "_Tensor") -> "_Tensor":
        return add(self, (-1.0) * other)


class DenseTensor(_Tensor):
    """A dense column-major FP64 operand (the reference's ``Array``)."""

    kind = 0

    def __init__(self, array: Optional[np.ndarray] = None, ctx: Optional[Context] = None, *, dims=None,
                 _handle=None):
        ctx = ctx or default_context()
        if _handle is not None:
            super().__init__(ctx, _handle)
            return
        if array is None:
            dims = tuple(int(d) for d in dims)
            data = None
        else:
            a = np.asarray(array, dtype=np.float64)
            dims = a.shape
            data = np.asfortranarray(a).reshape(-1, order="F")
            data = np.ascontiguousarray(data)
        h = C.c_void_p()
        _check(ctx, ctx._lib.sb_tensor_create_dense(ctx._h, len(dims), _i64(dims), _f64ptr(data), C.byref(h)))
        super().__init__(ctx, h)

    @staticmethod
    def from_device(ptr: int, dims: Sequence[int], ctx: Optional[Context] = None) -> "DenseTensor":
        ctx = ctx or default_context()
        h = C.c_void_p()
        _check(ctx, ctx._lib.sb_tensor_create_dense_device(ctx._h, len(dims), _i64(dims), C.c_void_p(ptr), C.byref(h)))
        return DenseTensor(ctx=ctx, _handle=h)

    def to_numpy(self) -> np.ndarray:
        dims = self.dims
        n = int(np.prod(dims)) if dims else 1
        out = np.empty(n, dtype=np.float64)
        _check(self.ctx, self.ctx._lib.sb_tensor_export_dense(self.ctx._h, self._h, _f64ptr(out)))
        return out.reshape(dims, order="F") if dims else out.reshape(())


class NewBlockSparseSorted(_Tensor):
    """Prefix-sparse / tail-dense block store (``src/blocksparse/storage.jl:3-9``).

    ``keys``: list of 1-based prefix tuples; ``ids``: 1-based slot of each key's
    payload in ``data`` (default ``1..n``); ``data``: concatenated column-major
    blocks.  Keys are kept sorted column-major on the device side.
    """

    kind = 2

    def __init__(self, dims: Sequence[int], n2: int, keys: Optional[Sequence[Sequence[int]]] = None,
                 ids: Optional[Sequence[int]] = None, data: Optional[np.ndarray] = None,
                 ctx: Optional[Context] = None, _handle=None, block_dims: Optional[Sequence[Sequence[int]]] = None):
        """With ``block_dims`` (one tail-extent tuple per key, same order as
        ``keys``) the tensor is ragged: each block is stored unpadded, column-
        major over its own extents, concatenated in ``keys`` order."""
        ctx = ctx or default_context()
        if _handle is not None:
            super().__init__(ctx, _handle)
            return
        dims = tuple(int(d) for d in dims)
        P = len(dims) - n2
        keys = [tuple(k) for k in (keys or [])]
        if P == 0 and data is not None and not keys:
            keys = [()] if np.asarray(data).size else []
        n = len(keys)
        flat = [int(x) for k in keys for x in k]
        d = None if data is None else np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(-1))
        h = C.c_void_p()
        if block_dims is not None:
            bd = [int(x) for b in block_dims for x in b]
            _check(ctx, ctx._lib.sb_tensor_create_bs_ragged(ctx._h, len(dims), _i64(dims), int(n2), n, _i64(flat),
                                                            _i64(bd), _f64ptr(d), C.byref(h)))
        else:
            _check(ctx, ctx._lib.sb_tensor_create_bs(ctx._h, len(dims), _i64(dims), int(n2), n, _i64(flat),
                                                     _i64(ids) if ids is not None else None, _f64ptr(d), C.byref(h)))
        super().__init__(ctx, h)

    def _layout(self):
        i = self._info()
        n, n2 = i["nkeys"], i["n2"]
        rg, ln = C.c_int(), C.c_int64()
        bd = (C.c_int64 * max(n * n2, 1))()
        _check(self.ctx, self.ctx._lib.sb_tensor_block_dims(self._h, C.byref(rg), bd, C.byref(ln)))
        return bool(rg.value), [tuple(bd[j * n2 + t] for t in range(n2)) for j in range(n)], ln.value

    @property
    def is_ragged(self) -> bool:
        return self._layout()[0]

    @property
    def block_dims(self) -> List[Tuple[int, ...]]:
        """Tail extents of every block in key order (the full tail dims when uniform)."""
        return self._layout()[1]

    @property
    def n2(self) -> int:
        return self._info()["n2"]

    @property
    def P(self) -> int:
        i = self._info()
        return len(i["dims"]) - i["n2"]

    @property
    def blksize(self) -> int:
        return self._info()["blksize"]

    def _export(self, with_data: bool = True):
        """(keys, ids, payload); without ``with_data`` the payload is None and
        nothing is copied from the device (keys live on the host)."""
        i = self._info()
        P, n = len(i["dims"]) - i["n2"], i["nkeys"]
        keys = (C.c_int64 * max(n * P, 1))()
        ids = (C.c_int64 * max(n, 1))()
        data = None
        if with_data:
            _, _, plen = self._layout()
            data = np.empty(plen, dtype=np.float64)
        _check(self.ctx, self.ctx._lib.sb_tensor_export_bs(self.ctx._h, self._h, keys, ids, _f64ptr(data)))
        klist = [tuple(keys[j * P + t] for t in range(P)) for j in range(n)]
        return klist, [ids[j] for j in range(n)], data

    @property
    def keys(self) -> List[Tuple[int, ...]]:
        return self._export(with_data=False)[0]

    @property
    def ids(self) -> List[int]:
        return self._export(with_data=False)[1]

    @property
    def data(self) -> np.ndarray:
        return self._export()[2]

    def blocks_by_key(self) -> dict:
        """Flat column-major payload of every block (unpadded when ragged)."""
        keys, ids, data = self._export()
        _, bd, _ = self._layout()
        out, off = {}, 0
        for k, e in zip(keys, bd):
            ln = int(np.prod(e)) if e else 1
            out[k] = data[off: off + ln].copy()
            off += ln
        return out

    @staticmethod
    def empty(dims: Sequence[int], n2: int, ctx: Optional[Context] = None,
              f32: bool = False) -> "NewBlockSparseSorted":
        """``NewBlockSparseSorted{T,N,N2}(dims)`` (storage.jl:86-93).  With
        ``f32`` the tensor stores FP32 values (sb_tensor_create_bs_f32): an
        output for tensor-core contractions, e.g. H_eff chain intermediates."""
        if not f32:
            return NewBlockSparseSorted(dims, n2, ctx=ctx)
        ctx = ctx or default_context()
        dims = tuple(int(d) for d in dims)
        h = C.c_void_p()
        _check(ctx, ctx._lib.sb_tensor_create_bs_f32(ctx._h, len(dims), _i64(dims), int(n2), C.byref(h)))
        return NewBlockSparseSorted(dims, n2, ctx=ctx, _handle=h)

    @property
    def is_f32(self) -> bool:
        """FP32 storage (values widened to FP64 on export)."""
        v = C.c_int()
        _check(self.ctx, self.ctx._lib.sb_tensor_storage_f32(self._h, C.byref(v)))
        return bool(v.value)


class COOTensor(_Tensor):
    """Coordinate tensor (``src/coo/storage.jl:1-6``)."""

    kind = 1

    def __init__(self, dims: Sequence[int], keys: Optional[Sequence[Sequence[int]]] = None,
                 vals: Optional[Sequence[float]] = None, dirty: bool = False, ctx: Optional[Context] = None,
                 _handle=None):
        ctx = ctx or default_context()
        if _handle is not None:
            super().__init__(ctx, _handle)
            return
        dims = tuple(int(d) for d in dims)
        keys = [tuple(k) for k in (keys or [])]
        v = np.ascontiguousarray(np.asarray(vals if vals is not None else [], dtype=np.float64))
        h = C.c_void_p()
        _check(ctx, ctx._lib.sb_tensor_create_coo(ctx._h, len(dims), _i64(dims), len(keys),
                                                  _i64([x for k in keys for x in k]), _f64ptr(v), int(dirty),
                                                  C.byref(h)))
        super().__init__(ctx, h)

    def _export(self):
        i = self._info()
        N, n = len(i["dims"]), i["nkeys"]
        keys = (C.c_int64 * max(n * N, 1))()
        vals = np.empty(n, dtype=np.float64)
        _check(self.ctx, self.ctx._lib.sb_tensor_export_coo(self.ctx._h, self._h, keys, _f64ptr(vals)))
        return [tuple(keys[j * N + t] for t in range(N)) for j in range(n)], vals

    @property
    def keys(self):
        return self._export()[0]

    @property
    def vals(self):
        return list(self._export()[1])

    @property
    def dirty(self) -> bool:
        return self._info()["dirty"]


class AliasedBlockSparse(_Tensor):
    """Template-aliased block store (``src/aliased/storage.jl:46-54``)."""

    kind = 3

    def __init__(self, dims: Sequence[int], n2: int, templates: Optional[np.ndarray] = None,
                 keys: Optional[Sequence[Sequence[int]]] = None, alias_ids: Optional[Sequence[int]] = None,
                 scalars: Optional[Sequence[float]] = None, ctx: Optional[Context] = None, _handle=None):
        ctx = ctx or default_context()
        if _handle is not None:
            super().__init__(ctx, _handle)
            return
        dims = tuple(int(d) for d in dims)
        P = len(dims) - n2
        blk = int(np.prod(dims[P:]))
        t = np.ascontiguousarray(np.asarray(templates if templates is not None else [], dtype=np.float64).reshape(-1))
        ntm = t.size // blk if blk else 0
        keys = [tuple(k) for k in (keys or [])]
        sc = np.ascontiguousarray(np.asarray(scalars if scalars is not None else [], dtype=np.float64))
        h = C.c_void_p()
        _check(ctx, ctx._lib.sb_tensor_create_aliased(ctx._h, len(dims), _i64(dims), int(n2), ntm, _f64ptr(t),
                                                      len(keys), _i64([x for k in keys for x in k]),
                                                      _i64(alias_ids or []), _f64ptr(sc), C.byref(h)))
        super().__init__(ctx, h)

    def _export(self, with_templates: bool = True):
        """(templates, keys, alias_ids, scalars); without ``with_templates``
        the templates are None and not copied from the device."""
        i = self._info()
        P, n, blk, ntm = len(i["dims"]) - i["n2"], i["nkeys"], i["blksize"], i["n_templates"]
        tm = np.empty(ntm * blk, dtype=np.float64) if with_templates else None
        keys = (C.c_int64 * max(n * P, 1))()
        aids = (C.c_int64 * max(n, 1))()
        sc = np.empty(n, dtype=np.float64)
        _check(self.ctx, self.ctx._lib.sb_tensor_export_aliased(self.ctx._h, self._h, _f64ptr(tm), keys, aids,
                                                                _f64ptr(sc)))
        return tm, [tuple(keys[j * P + t] for t in range(P)) for j in range(n)], [aids[j] for j in range(n)], sc

    @property
    def n_templates(self) -> int:
        return self._info()["n_templates"]

    @property
    def blksize(self) -> int:
        return self._info()["blksize"]

    @property
    def keys(self):
        return self._export(with_templates=False)[1]

    def logical_blocks(self) -> dict:
        """Per-key ``scalar * template`` (the unit the reference's tests compare)."""
        tm, keys, aids, sc = self._export()
        blk = self.blksize
        return {k: s * tm[(a - 1) * blk: a * blk] for k, a, s in zip(keys, aids, sc)}

    @staticmethod
    def empty(dims: Sequence[int], n2: int, ctx: Optional[Context] = None) -> "AliasedBlockSparse":
        return AliasedBlockSparse(dims, n2, ctx=ctx)


def to_uniform(A: NewBlockSparseSorted) -> NewBlockSparseSorted:
    """Zero-pad a ragged tensor to the reference's uniform block format."""
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_tensor_to_uniform(A.ctx._h, A._h, C.byref(h)))
    return _from_handle(A.ctx, h)


def to_ragged(A: NewBlockSparseSorted, block_dims: Sequence[Sequence[int]], check_zero: bool = True):
    """Crop every block of a uniform tensor to ``block_dims`` (key order)."""
    bd = [int(x) for b in block_dims for x in b]
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_tensor_to_ragged(A.ctx._h, A._h, _i64(bd), int(check_zero), C.byref(h)))
    return _from_handle(A.ctx, h)


def crop_padding(A: NewBlockSparseSorted) -> NewBlockSparseSorted:
    """The ragged tensor of A's blocks cropped to the smallest extents that keep
    their nonzero entries: the zero padding of the reference layout (every
    U(1) sector padded to the largest) removed without knowing the sectors."""
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_tensor_crop_padding(A.ctx._h, A._h, C.byref(h)))
    return _from_handle(A.ctx, h)


def compression_ratio(A: AliasedBlockSparse) -> float:
    """``compression_ratio`` (aliased/storage.jl:163-164)."""
    i = A._info()
    return 1.0 if i["n_templates"] == 0 else i["nkeys"] / i["n_templates"]


def _wrap(ctx: Context, h: C.c_void_p) -> _Tensor:
    kind = C.c_int()
    _check(ctx, ctx._lib.sb_tensor_info(h, C.byref(kind), None, None, None, None, None, None, None))
    cls = {0: DenseTensor, 1: COOTensor, 2: NewBlockSparseSorted, 3: AliasedBlockSparse}[kind.value]
    return cls.__new__(cls), cls


def _from_handle(ctx: Context, h: C.c_void_p) -> _Tensor:
    obj, cls = _wrap(ctx, h)
    _Tensor.__init__(obj, ctx, h)
    return obj


def _as_operand(x, ctx: Context) -> _Tensor:
    if isinstance(x, _Tensor):
        return x
    return DenseTensor(np.asarray(x, dtype=np.float64), ctx)


# ── vector-space operations (KrylovKit hooks, src/tensor_wrappers.jl:793-923) ──

MAP_AXPY, MAP_AXPBY, MAP_COPY, MAP_MUL = 0, 1, 2, 3


def norm(A: _Tensor) -> float:
    """``LinearAlgebra.norm(w)``: 2-norm of the stored values (aliased: of the
    logical blocks, tensor_wrappers_aliased.jl:524-536)."""
    out = C.c_double()
    _check(A.ctx, A.ctx._lib.sb_tensor_norm(A.ctx._h, A._h, C.byref(out)))
    return out.value


def dot(A: _Tensor, B: _Tensor) -> float:
    """``dot(x, y) = (dag(x) * y)[]`` for real tensors: the sum over keys in
    both operands of the block dot products (contract_bs_bs_to_dense! with every
    label shared)."""
    out = C.c_double()
    _check(A.ctx, A.ctx._lib.sb_tensor_dot(A.ctx._h, A._h, B._h, C.byref(out)))
    return out.value


inner = dot


def copy(A: _Tensor) -> _Tensor:
    """``copy(w)``: deep copy on the device."""
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_tensor_copy(A.ctx._h, A._h, C.byref(h)))
    return _from_handle(A.ctx, h)


def similar(A: _Tensor) -> _Tensor:
    """``similar(w)``: same keys and layout, zero values."""
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_tensor_similar(A.ctx._h, A._h, C.byref(h)))
    return _from_handle(A.ctx, h)


def scale_(A: _Tensor, alpha: float) -> _Tensor:
    """In place: stored values (aliased: scalars) times ``alpha``."""
    _check(A.ctx, A.ctx._lib.sb_tensor_scale(A.ctx._h, A._h, float(alpha)))
    return A


def fill_(A: _Tensor, x: float) -> _Tensor:
    """``fill!(w, x)`` on the stored values."""
    _check(A.ctx, A.ctx._lib.sb_tensor_fill(A.ctx._h, A._h, float(x)))
    return A


def map_(R: _Tensor, A: _Tensor, op: int, alpha: float = 1.0, beta: float = 1.0) -> _Tensor:
    """``map!(f, R, R, A)`` by stored position for f in MAP_AXPY (r + alpha*a),
    MAP_AXPBY (beta*r + alpha*a), MAP_COPY (a), MAP_MUL (r*a)."""
    _check(R.ctx, R.ctx._lib.sb_tensor_map(R.ctx._h, R._h, A._h, int(op), float(alpha), float(beta)))
    return R


def axpy_(alpha: float, x: _Tensor, y: _Tensor) -> _Tensor:
    """``y .= y .+ alpha .* x`` (same sparsity pattern)."""
    return map_(y, x, MAP_AXPY, alpha)


def axpby_(alpha: float, x: _Tensor, beta: float, y: _Tensor) -> _Tensor:
    """``y .= beta .* y .+ alpha .* x`` (same sparsity pattern)."""
    return map_(y, x, MAP_AXPBY, alpha, beta)


def add(A: _Tensor, B: _Tensor) -> _Tensor:
    """``x + y``: union of the block keys; shared keys add."""
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_tensor_add(A.ctx._h, A._h, B._h, C.byref(h)))
    return _from_handle(A.ctx, h)


def fuse_axes(A: _Tensor, ax1: int, ax2: int) -> _Tensor:
    """``fuse_two_axes!`` (block-sparse, conversions.jl:228-314) or
    ``fuse_axes_coo`` (COO, coo/conversions.jl:174-222); axes 1-based."""
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_fuse_axes(A.ctx._h, A._h, int(ax1), int(ax2), C.byref(h)))
    return _from_handle(A.ctx, h)


# ── block factorisations (src/ops_factorize.jl) ────────────────────────────

def is_dense(A: _Tensor) -> bool:
    """``is_dense(A)`` (src/blocksparse/storage.jl:413-425): every prefix
    combination has a block."""
    v = C.c_int()
    _check(A.ctx, A.ctx._lib.sb_tensor_is_dense(A._h, C.byref(v)))
    return bool(v.value)


def blocksparse_left_qr(A: NewBlockSparseSorted):
    """``blocksparse_left_qr(A)`` (ops_factorize.jl:8-43) for A with prefix
    (l, r) and dense tail (s).  Returns (Q, R, l_vals, r_vals): Q block-sparse
    (l | s, b), R a DenseTensor k x n_r, the sorted distinct l and r values."""
    ctx = A.ctx
    dims = A.dims
    q, r = C.c_void_p(), C.c_void_p()
    lv = (C.c_int64 * max(dims[0], 1))()
    rv = (C.c_int64 * max(dims[1], 1))()
    nl, nr = C.c_int64(), C.c_int64()
    _check(ctx, ctx._lib.sb_blocksparse_left_qr(ctx._h, A._h, C.byref(q), C.byref(r), lv, C.byref(nl), rv,
                                                C.byref(nr)))
    return (_from_handle(ctx, q), _from_handle(ctx, r), [lv[i] for i in range(nl.value)],
            [rv[i] for i in range(nr.value)])


def blocksparse_svd(A: NewBlockSparseSorted, ortho: str = "left", maxdim: int = 2 ** 62, mindim: int = 1,
                    cutoff: float = 0.0):
    """``blocksparse_svd(A; ortho, maxdim, mindim, cutoff)`` (ops_factorize.jl:50-148)
    for A with prefix (L, R) and dense tail (s1, s2).  Returns
    (U, SV, svs_kept, spectrum) with spectrum = {"eigs": svs^2, "truncerr": ...}."""
    if ortho not in ("left", "right"):
        raise ValueError("ortho must be 'left' or 'right'")
    ctx = A.ctx
    dims = A.dims
    cap = max(dims[0] * dims[2], 1)
    u, sv = C.c_void_p(), C.c_void_p()
    svs = np.zeros(cap)
    nk, te = C.c_int64(), C.c_double()
    _check(ctx, ctx._lib.sb_blocksparse_svd(ctx._h, A._h, int(ortho == "right"), int(maxdim), int(mindim),
                                            float(cutoff), C.byref(u), C.byref(sv), _f64ptr(svs), cap,
                                            C.byref(nk), C.byref(te)))
    kept = svs[: nk.value].copy()
    return _from_handle(ctx, u), _from_handle(ctx, sv), kept, {"eigs": kept ** 2, "truncerr": te.value}


def contract_(C_: _Tensor, labelsC: Sequence[Any], A, labelsA: Sequence[Any], B, labelsB: Sequence[Any]) -> _Tensor:
    """``contract!(C, labelsC, A, labelsA, B, labelsB)``: overwrite ``C`` with A·B.

    Dispatches like ``src/tensoralgebra/contract.jl:37-104``: one reduced
    shared label goes to the single-label kernel of the (C, A, B) storage
    combination, otherwise to ``contract_shared!``.  ``B`` may be a numpy
    array (uploaded as a dense operand).
    """
    ctx = C_.ctx
    A = _as_operand(A, ctx)
    B = _as_operand(B, ctx)
    lc, nc = _labels(labelsC)
    la, na = _labels(labelsA)
    lb, nb = _labels(labelsB)
    _check(ctx, ctx._lib.sb_contract(ctx._h, C_._h, lc, nc, A._h, la, na, B._h, lb, nb))
    return C_


def contract_bs_bs_to_dense(dimsC: Sequence[int], labelsC, A: NewBlockSparseSorted, labelsA,
                            B: NewBlockSparseSorted, labelsB) -> DenseTensor:
    """``contract_bs_bs_to_dense!`` (contract_bs_bs.jl:736-754): P_C = 0 sink."""
    Cd = DenseTensor(ctx=A.ctx, dims=dimsC)
    contract_(Cd, labelsC, A, labelsA, B, labelsB)
    return Cd


def blocksparse_from_dense(A, n2: int, atol: float = 0.0, rtol: float = 0.0, dropzeros: bool = True,
                           ctx: Optional[Context] = None) -> NewBlockSparseSorted:
    ctx = ctx or (A.ctx if isinstance(A, _Tensor) else default_context())
    D = _as_operand(A, ctx)
    h = C.c_void_p()
    _check(ctx, ctx._lib.sb_blocksparse_from_dense(ctx._h, D._h, int(n2), float(atol), float(rtol), int(dropzeros),
                                                   C.byref(h)))
    return _from_handle(ctx, h)


def coo_from_dense(A, atol: float = 1e-12, rtol: float = 0.0, ctx: Optional[Context] = None) -> COOTensor:
    ctx = ctx or (A.ctx if isinstance(A, _Tensor) else default_context())
    D = _as_operand(A, ctx)
    h = C.c_void_p()
    _check(ctx, ctx._lib.sb_coo_from_dense(ctx._h, D._h, float(atol), float(rtol), C.byref(h)))
    return _from_handle(ctx, h)


def to_dense(A: _Tensor) -> np.ndarray:
    """Materialise any storage as a numpy array (computed on the device)."""
    if isinstance(A, DenseTensor):
        return A.to_numpy()
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_to_dense(A.ctx._h, A._h, C.byref(h)))
    return _from_handle(A.ctx, h).to_numpy()


def to_blocksparse(A: AliasedBlockSparse) -> NewBlockSparseSorted:
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_aliased_to_blocksparse(A.ctx._h, A._h, C.byref(h)))
    return _from_handle(A.ctx, h)


def permutedims(A: _Tensor, perm: Sequence[int]) -> _Tensor:
    """1-based ``perm`` as in Julia; returns a new tensor."""
    arr = (C.c_int * max(len(perm), 1))(*[int(p) for p in perm])
    h = C.c_void_p()
    _check(A.ctx, A.ctx._lib.sb_permutedims(A.ctx._h, A._h, arr, C.byref(h)))
    return _from_handle(A.ctx, h)


def sort_(A: COOTensor) -> COOTensor:
    """``sort!(::COOTensor)`` → ``sort_coo!`` (coo/storage.jl:182-196)."""
    _check(A.ctx, A.ctx._lib.sb_coo_sort(A.ctx._h, A._h))
    return A


def output_inds(indsA: Sequence[Any], indsB: Sequence[Any], denseA: Iterable[Any], denseB: Iterable[Any],
                is_link=lambda i: False, link_level=lambda i: 0):
    """Output index order of ``output_inds`` (src/tensor_wrappers.jl:477-526).

    Returns ``(indsC, dense_tail)``: unique indices of A then of B, bucketed as
    [sparse links sorted by ``link_level``, sparse non-links, dense tail].
    """
    setA, setB = set(indsA), set(indsB)
    dA, dB = set(denseA), set(denseB)
    sparse_link, sparse_nonlink, dense_tail = [], [], []

    def push(i):
        if i in dA or i in dB:
            dense_tail.append(i)
        elif is_link(i):
            sparse_link.append(i)
        else:
            sparse_nonlink.append(i)

    for i in indsA:
        if i not in setB:
            push(i)
    for i in indsB:
        if i not in setA:
            push(i)
    sparse_link.sort(key=link_level)
    return tuple(sparse_link + sparse_nonlink + dense_tail), dense_tail
