"""Failure path of the bounded device waits (through the C ABI).

Every mbarrier wait of the tensor-core M2L kernel gives up after a limit,
sets the FMM's error flag and lets the kernel drain and return; the host
turns the flag into NNK_E_TIMEOUT.  nnk_fmm_test_wait_timeout runs that
kernel once with its threads first waiting, for a short limit, on a barrier
that nothing completes: no copy or MMA is issued, the kernel frees its
tensor memory and returns.  The call must report NNK_E_TIMEOUT, and the same
FMM (same context) must then evaluate normally.  Nothing here faults, traps
or waits without a bound."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def fixture_fmm(precision):
    g = np.load(os.path.join(GOLDEN, "adaptive_nearest_1200.npz"))
    NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
    t = nk.OcTree(g["coarse"], g["coarse"], nodeCapacity=int(g["cap"]), nearest=1, finePoints=g["fine"], NN=NN)
    return g, t, nk.KIFMM(t, [float(g["eps"]), float(g["mu"])], precision=precision)


def test_bounded_wait_gives_up_and_the_fmm_recovers():
    L = nk._lib
    g, t, fmm = fixture_fmm("mixed")
    st = fmm.stats()
    assert st["m2l_rank"] == 256 and st["m2l_pairs"] > 0
    before = fmm.computeVel(g["F"])
    for polls in (1000, 20000):  # twice in a row: the flag is cleared once reported
        rc = L.lib.nnk_fmm_test_wait_timeout(fmm.h, polls)
        assert rc == L.NNK_E_TIMEOUT
        assert "bounded wait" in L.lib.nnk_last_error(fmm.ctx.h).decode()
        after = fmm.computeVel(g["F"])
        assert np.array_equal(after, before)  # the M2L adds its partial blocks in a fixed order


def test_probe_needs_the_tensor_core_m2l():
    L = nk._lib
    g, t, fmm = fixture_fmm("fp64")
    assert L.lib.nnk_fmm_test_wait_timeout(fmm.h, 1000) == L.NNK_E_STATE
    assert L.lib.nnk_fmm_test_wait_timeout(fmm.h, 0) == L.NNK_E_ARG
    v = fmm.computeVel(g["F"])
    assert rel(v, g["vel"]) <= 1e-6
