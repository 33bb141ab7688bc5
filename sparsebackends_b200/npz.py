"""``.npz`` interchange of stored tensors in the reference's own layout.

One file holds one tensor as the fields of the reference's storage types, so a
Julia run can dump its operands (e.g. with NPZ.jl) and feed the GPU path, and
the GPU path's results can be compared back:

* block-sparse ``NewBlockSparseSorted`` (src/blocksparse/storage.jl:3-9):
  ``dims``, ``n2``, ``blksize``, ``keys`` (n x P, 1-based), ``ids`` (1-based
  slots), ``data`` (blocks concatenated column-major by slot); ragged tensors
  add ``block_dims`` (n x n2) and store ``data`` unpadded in key order;
* COO ``COOTensor`` (src/coo/storage.jl:1-6): ``dims``, ``keys`` (n x N),
  ``vals``, ``dirty``;
* aliased ``AliasedBlockSparse`` (src/aliased/storage.jl:46-54): ``dims``,
  ``n2``, ``templates``, ``keys``, ``alias_ids``, ``scalars``;
* dense: ``dims``, ``data`` (column-major).

Every file carries ``format`` = "sparsebackends-npz", ``version`` = 1 and
``kind``.  Integers are int64, values float64.  ``read_npz`` / ``write_npz``
are host-only; ``save`` / ``load`` move tensors between a file and the device.
"""
from __future__ import annotations

from typing import Any, Dict, Optional

import numpy as np

FORMAT = "sparsebackends-npz"
VERSION = 1
KINDS = ("dense", "coo", "blocksparse", "aliased")


def _i64(x, shape=None):
    a = np.asarray(x, dtype=np.int64)
    return a.reshape(shape) if shape is not None else a


def write_npz(path: str, kind: str, **fields: Any) -> None:
    """Write one tensor's fields (see the module docstring for the names)."""
    if kind not in KINDS:
        raise ValueError(f"unknown kind {kind!r}")
    out: Dict[str, np.ndarray] = {"format": np.array(FORMAT), "version": np.array(VERSION, dtype=np.int64),
                                  "kind": np.array(kind)}
    dims = _i64(fields["dims"])
    out["dims"] = dims
    N = len(dims)
    if kind == "dense":
        out["data"] = np.asarray(fields["data"], dtype=np.float64).reshape(-1, order="F") \
            if np.ndim(fields["data"]) > 1 else np.asarray(fields["data"], dtype=np.float64)
    elif kind == "coo":
        keys = [tuple(k) for k in fields.get("keys", [])]
        out["keys"] = _i64(keys, (len(keys), N))
        out["vals"] = np.asarray(fields.get("vals", []), dtype=np.float64)
        out["dirty"] = np.array(bool(fields.get("dirty", False)))
    elif kind == "blocksparse":
        n2 = int(fields["n2"])
        P = N - n2
        keys = [tuple(k) for k in fields.get("keys", [])]
        n = len(keys)
        out["n2"] = np.array(n2, dtype=np.int64)
        out["blksize"] = np.array(int(np.prod(dims[P:])), dtype=np.int64)
        out["keys"] = _i64(keys, (n, P))
        ids = fields.get("ids")
        out["ids"] = _i64(ids if ids is not None else np.arange(1, n + 1))
        out["data"] = np.asarray(fields.get("data", []), dtype=np.float64).reshape(-1)
        if fields.get("block_dims") is not None:
            out["block_dims"] = _i64([tuple(b) for b in fields["block_dims"]], (n, n2))
    else:
        n2 = int(fields["n2"])
        P = N - n2
        keys = [tuple(k) for k in fields.get("keys", [])]
        out["n2"] = np.array(n2, dtype=np.int64)
        out["templates"] = np.asarray(fields.get("templates", []), dtype=np.float64).reshape(-1)
        out["keys"] = _i64(keys, (len(keys), P))
        out["alias_ids"] = _i64(fields.get("alias_ids", []))
        out["scalars"] = np.asarray(fields.get("scalars", []), dtype=np.float64)
    np.savez(path, **out)


def read_npz(path: str) -> Dict[str, Any]:
    """Read a file written by write_npz (or by any writer of the same fields)."""
    with np.load(path, allow_pickle=False) as z:
        if str(z["format"]) != FORMAT:
            raise ValueError(f"{path}: not a {FORMAT} file")
        if int(z["version"]) != VERSION:
            raise ValueError(f"{path}: unsupported version {int(z['version'])}")
        kind = str(z["kind"])
        d: Dict[str, Any] = {"kind": kind, "dims": tuple(int(x) for x in z["dims"])}
        if kind == "dense":
            d["data"] = z["data"].copy()
        elif kind == "coo":
            d["keys"] = [tuple(int(x) for x in r) for r in z["keys"]]
            d["vals"] = z["vals"].copy()
            d["dirty"] = bool(z["dirty"])
        elif kind == "blocksparse":
            d["n2"] = int(z["n2"])
            d["blksize"] = int(z["blksize"])
            d["keys"] = [tuple(int(x) for x in r) for r in z["keys"]]
            d["ids"] = [int(x) for x in z["ids"]]
            d["data"] = z["data"].copy()
            d["block_dims"] = [tuple(int(x) for x in r) for r in z["block_dims"]] if "block_dims" in z else None
        elif kind == "aliased":
            d["n2"] = int(z["n2"])
            d["templates"] = z["templates"].copy()
            d["keys"] = [tuple(int(x) for x in r) for r in z["keys"]]
            d["alias_ids"] = [int(x) for x in z["alias_ids"]]
            d["scalars"] = z["scalars"].copy()
        else:
            raise ValueError(f"{path}: unknown kind {kind!r}")
        return d


def save(path: str, T) -> None:
    """Write a device tensor (exported in the reference layout: keys sorted
    column-major, ids = 1:n)."""
    import sparsebackends_b200 as sb
    if isinstance(T, sb.NewBlockSparseSorted):
        ragged = T.is_ragged
        write_npz(path, "blocksparse", dims=T.dims, n2=T.n2, keys=T.keys, ids=T.ids, data=T.data,
                  block_dims=T.block_dims if ragged else None)
    elif isinstance(T, sb.COOTensor):
        write_npz(path, "coo", dims=T.dims, keys=T.keys, vals=T.vals, dirty=T.dirty)
    elif isinstance(T, sb.AliasedBlockSparse):
        tmpl, keys, alias, scal = T._export()
        write_npz(path, "aliased", dims=T.dims, n2=T._info()["n2"], templates=tmpl, keys=keys, alias_ids=alias,
                  scalars=scal)
    elif isinstance(T, sb.DenseTensor):
        write_npz(path, "dense", dims=T.dims, data=T.to_numpy())
    else:
        raise TypeError(f"cannot save {type(T).__name__}")


def load(path: str, ctx: Optional[Any] = None):
    """Read a file onto the device as the matching tensor type."""
    import sparsebackends_b200 as sb
    d = read_npz(path)
    k = d["kind"]
    if k == "blocksparse":
        return sb.NewBlockSparseSorted(d["dims"], d["n2"], d["keys"], None if d["block_dims"] else d["ids"],
                                       d["data"], ctx=ctx, block_dims=d["block_dims"])
    if k == "coo":
        return sb.COOTensor(d["dims"], d["keys"], d["vals"], dirty=d["dirty"], ctx=ctx)
    if k == "aliased":
        return sb.AliasedBlockSparse(d["dims"], d["n2"], d["templates"], d["keys"], d["alias_ids"], d["scalars"],
                                     ctx=ctx)
    return sb.DenseTensor(np.asarray(d["data"]).reshape(d["dims"], order="F"), ctx)
