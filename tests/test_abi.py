"""C-ABI checks that need no GPU: the library builds, loads and exports every
symbol declared in include/sparseb.h; without a CUDA device every entry point
fails loudly with a status code instead of falling back to the CPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sparseb.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"SB_API\s+[\w\s\*]+?\b(sb_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "sb_contract" in syms and "sb_ctx_create" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol():
    from sparsebackends_b200 import _lib
    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
    # the ctypes signature table covers every declared symbol too
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_every_kernel_source_compiles_for_sm100a():
    from sparsebackends_b200 import build
    lib = build.build()
    assert os.path.exists(lib)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_no_gpu_fails_loudly():
    import sparsebackends_b200 as sb
    with pytest.raises(sb.SparseBackendsError) as ei:
        sb.Context(0)
    assert ei.value.status in ("SB_ERR_CUDA", "SB_ERR_INVALID_ARG")


def test_null_arguments_are_rejected_without_touching_the_gpu():
    from sparsebackends_b200 import _lib
    lib = _lib.load()
    assert lib.sb_ctx_create(0, 0, None) == 1  # SB_ERR_INVALID_ARG
    assert lib.sb_tensor_info(None, None, None, None, None, None, None, None, None) == 1
    assert lib.sb_contract(None, None, None, 0, None, None, 0, None, None, 0) == 1
    assert lib.sb_ctx_destroy(None) == 0
    assert lib.sb_tensor_free(None) == 0


def test_label_key_mapping():
    import sparsebackends_b200 as sb
    assert sb.label_key((7, 1)) == (7, 1)
    a, b = sb.label_key("r"), sb.label_key("r")
    assert a == b and a[1] == 0
    assert sb.label_key("r") != sb.label_key("i")


def test_packed_labels_cache_is_exact():
    """String-label lists are packed once and reused; every other label list
    is packed afresh; both give the words of label_key."""
    import sparsebackends_b200 as sb

    def words(labels):
        return [w for l in labels for w in sb.label_key(l)]

    strs = ["ql", "s1", "s2", "qr", "ml", "mr"]
    a1, n1 = sb._labels(strs)
    a2, n2 = sb._labels(list(strs))
    assert a1 is a2 and n1 == n2 == 6 and list(a1) == words(strs)
    mixed = ["ql", (7, 1), 3]
    b1, _ = sb._labels(mixed)
    b2, _ = sb._labels(mixed)
    assert b1 is not b2 and list(b1) == list(b2) == words(mixed)
    # equal-comparing labels of different types keep their own words
    assert list(sb._labels([1])[0]) != list(sb._labels([1.0])[0])


def test_output_inds_order():
    """output_inds (src/tensor_wrappers.jl:477-526): links by level, non-links, dense tail."""
    import sparsebackends_b200 as sb
    level = {"l2": 2, "l1": 1}
    inds, dense = sb.output_inds(["s1", "l2", "x", "w"], ["w", "l1", "y"], denseA={"x"}, denseB={"y"},
                                 is_link=lambda i: i in level, link_level=lambda i: level.get(i, 0))
    assert inds == ("l1", "l2", "s1", "x", "y")
    assert dense == ["x", "y"]
