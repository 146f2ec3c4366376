"""The C ABI library loads, exports every symbol include/nnkifmm.h declares,
and refuses FMM work without a GPU (no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

import nnkifmm as nk
from conftest import ROOT


def header_symbols():
    src = open(os.path.join(ROOT, "include", "nnkifmm.h")).read()
    return sorted(set(re.findall(r"\b(nnk_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(nk.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    from nnkifmm._lib import SIGNATURES
    assert set(header_symbols()) == set(SIGNATURES)


def test_version_string():
    assert nk.lib.nnk_version().decode().startswith("nnkifmm")


def test_fmm_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    x = np.random.default_rng(0).random((50, 3))
    t = nk.OcTree(x, x, nodeCapacity=10)
    with pytest.raises(nk.NNKError, match="no CUDA device"):
        nk.KIFMM(t, [1e-3, 1.0])


def test_batch_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from nnkifmm.batch import BatchMobility
    x = np.random.default_rng(1).random((40, 3))
    f = np.random.default_rng(2).random((120, 3))
    with pytest.raises(nk.NNKError, match="no CUDA device"):
        BatchMobility([(x, f)], [1e-3, 1.0], cap=10, precision="fp64", nrhs=2)


def test_context_outlives_its_handles_in_any_order():
    """A tree keeps its context alive: destroying the context first, then
    using and destroying the tree, is safe (C ABI, host builder)."""
    L = nk._lib
    ctx = ctypes.c_void_p()
    assert L.lib.nnk_ctx_create(0, ctypes.byref(ctx)) == L.NNK_OK
    x = np.ascontiguousarray(np.random.default_rng(3).random((200, 3)))
    params = L.TreeParams(20, 20, 0, 1)
    tree = ctypes.c_void_p()
    rc = L.lib.nnk_tree_build(ctx, L.ptr(x), 200, L.ptr(x), 200, None, 0, None, None, None, ctypes.byref(params),
                              ctypes.byref(tree))
    assert rc == L.NNK_OK
    assert L.lib.nnk_ctx_destroy(ctx) == L.NNK_OK
    info = L.TreeInfo()
    assert L.lib.nnk_tree_info_get(tree, ctypes.byref(info)) == L.NNK_OK
    assert info.num_points == 200
    assert L.lib.nnk_tree_destroy(tree) == L.NNK_OK


def test_malformed_nearest_matrix_rejected():
    """A caller's NN CSR is checked before it is read: row pointers that do
    not start at 0 or decrease, columns outside potPoints and missing arrays
    return NNK_E_ARG with a message (C ABI, host builder)."""
    L = nk._lib
    ctx = ctypes.c_void_p()
    assert L.lib.nnk_ctx_create(0, ctypes.byref(ctx)) == L.NNK_OK
    rng = np.random.default_rng(4)
    x = np.ascontiguousarray(rng.random((100, 3)))
    f = np.ascontiguousarray(rng.random((3, 3)))
    params = L.TreeParams(20, 20, 1, 1)

    def build(rowptr, col, val):
        tree = ctypes.c_void_p()
        rp = np.ascontiguousarray(rowptr, np.int64)
        c = None if col is None else np.ascontiguousarray(col, np.int32)
        v = None if val is None else np.ascontiguousarray(val, np.float64)
        rc = L.lib.nnk_tree_build(ctx, L.ptr(x), 100, L.ptr(x), 100, L.ptr(f), 3, L.ptr(rp),
                                  None if c is None else L.ptr(c), None if v is None else L.ptr(v),
                                  ctypes.byref(params), ctypes.byref(tree))
        if rc == L.NNK_OK:
            L.lib.nnk_tree_destroy(tree)
        return rc, L.lib.nnk_last_error(ctx).decode()

    assert build([0, 1, 2, 3], [5, 6, 7], [1.0, 1.0, 1.0])[0] == L.NNK_OK
    assert build([0, 1, 3, 3], [5, 7, 6], [1.0, 0.5, 0.5])[0] == L.NNK_OK  # unsorted row: sorted
    assert build([0, 100, 2, 3], [5, 6, 7], [1.0] * 3) == (L.NNK_E_ARG, "bad NN rowptr")
    assert build([1, 1, 2, 3], [5, 6, 7], [1.0] * 3) == (L.NNK_E_ARG, "bad NN rowptr")
    assert build([0, 1, 2, 3], [5, 100, 7], [1.0] * 3) == (L.NNK_E_ARG, "NN column out of range")
    assert build([0, 1, 2, 3], [5, -1, 7], [1.0] * 3) == (L.NNK_E_ARG, "NN column out of range")
    assert build([0, 1, 2, 3], None, [1.0] * 3) == (L.NNK_E_ARG, "NN columns or values missing")
    assert L.lib.nnk_ctx_destroy(ctx) == L.NNK_OK
