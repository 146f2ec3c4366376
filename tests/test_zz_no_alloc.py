"""The allocation-free entry point nnk_direct_nearest_noalloc, through the C ABI.

Some callers cannot allocate device memory at call time (a MATLAB MEX
gateway whose device memory belongs to MATLAB's pool, a loop with a fixed
memory budget that must not pay cudaMalloc/cudaFree and their device
synchronization per step).  This entry point evaluates the NEAREST velocity by
direct summation using only caller-supplied device buffers plus a static
scratch array inside the library.  Here it is compared, on two calls in a row
with different forces, with the existing allocating entry point computeVel
(nnk_fmm_apply, FP64) on the 488-point rigid sphere, where the FMM is within 1e-5 of
the direct sum, and with the oracle's FP64 direct sum.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN
from nnkifmm import _lib as L

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_matches_computevel_twice():
    import torch
    g = np.load(os.path.join(GOLDEN, "sphere10_40.npz"))
    NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
    NN.sort_indices()
    eps, mu = float(g["eps"]), float(g["mu"])
    coarse, fine = g["coarse"], g["fine"]
    tree = nk.OcTree(coarse, coarse, nodeCapacity=int(g["cap"]), nearest=1, finePoints=fine, NN=NN)
    fmm = nk.KIFMM(tree, [eps, mu])
    dev = torch.device("cuda", 0)
    d = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    rowptr, col, val = d(NN.indptr, torch.int64), d(NN.indices, torch.int32), d(NN.data)
    dfine, dtgt = d(fine), d(coarse)
    vel = torch.empty((len(coarse), 3), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rng = np.random.default_rng(99)
    for call, F in enumerate([g["F"], rng.standard_normal(g["F"].shape)]):
        dF = d(F)
        rc = L.lib.nnk_direct_nearest_noalloc(0, stream, dF.data_ptr(), len(coarse), rowptr.data_ptr(),
                                              col.data_ptr(), val.data_ptr(), dfine.data_ptr(), len(fine),
                                              dtgt.data_ptr(), len(coarse), eps, mu, vel.data_ptr())
        assert rc == L.NNK_OK
        torch.cuda.synchronize()
        v = vel.cpu().numpy()
        v_fmm = fmm.computeVel(F)
        assert rel(v, v_fmm) <= 1e-4, (call, rel(v, v_fmm))
        if call == 0:
            assert rel(v, g["direct"]) <= 1e-12


def test_noalloc_rejects_too_many_fine_points():
    n = L.NOALLOC_MAX_FINE + 1
    rc = L.lib.nnk_direct_nearest_noalloc(0, None, 1, 1, 1, 1, 1, 1, n, 1, 1, 1e-3, 1.0, 1)
    assert rc == L.NNK_E_ARG


def test_noalloc_empty_inputs_and_bad_columns():
    """q = 0 gives zero velocities, m = 0 does nothing, and a column index
    outside [0, n) turns the velocities it reaches into NaN instead of reading
    out of bounds."""
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    d = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    rng = np.random.default_rng(5)
    F, tgt = d(rng.standard_normal((4, 3))), d(rng.random((3, 3)))
    vel = torch.full((3, 3), 7.0, dtype=torch.float64, device=dev)
    rp0 = d(np.zeros(1, np.int64), torch.int64)
    one = d(np.zeros(1, np.int32), torch.int32)
    rc = L.lib.nnk_direct_nearest_noalloc(0, stream, F.data_ptr(), 4, rp0.data_ptr(), one.data_ptr(),
                                          F.data_ptr(), F.data_ptr(), 0, tgt.data_ptr(), 3, 1e-3, 1.0,
                                          vel.data_ptr())
    assert rc == L.NNK_OK
    torch.cuda.synchronize()
    assert torch.count_nonzero(vel).item() == 0
    assert L.lib.nnk_direct_nearest_noalloc(0, stream, F.data_ptr(), 4, rp0.data_ptr(), one.data_ptr(),
                                            F.data_ptr(), F.data_ptr(), 0, None, 0, 1e-3, 1.0, None) == L.NNK_OK
    fine = d(rng.random((2, 3)))
    rp = d(np.array([0, 1, 2], np.int64), torch.int64)
    col = d(np.array([1, 4], np.int32), torch.int32)  # 4 is outside [0, 4)
    val = d(np.array([1.0, 1.0]))
    rc = L.lib.nnk_direct_nearest_noalloc(0, stream, F.data_ptr(), 4, rp.data_ptr(), col.data_ptr(),
                                          val.data_ptr(), fine.data_ptr(), 2, tgt.data_ptr(), 3, 1e-3, 1.0,
                                          vel.data_ptr())
    assert rc == L.NNK_OK
    torch.cuda.synchronize()
    assert torch.isnan(vel).all().item()
