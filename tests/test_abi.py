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
