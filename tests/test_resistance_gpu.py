"""Grand resistance matrix (Resistance/Gen_Resistance.m, Rigid_Resistance.m)
through the device FMM and GMRES: against the dense FP64 resistance problem,
and as the inverse of the mobility matrix of the same FMM operator."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN
from nnkifmm.batch import Body
from nnkifmm.resistance import force_moment, velocityModes
from oracle.kernel import kernel

pytestmark = pytest.mark.gpu


def sphere():
    g = np.load(os.path.join(GOLDEN, "sphere10_40.npz"))
    NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
    return g["coarse"], g["fine"], NN, float(g["eps"]), float(g["mu"])


@pytest.mark.parametrize("fmt", [1, 2])
def test_resistance_matrix_vs_dense_and_mobility(fmt):
    c, f, NN, eps, mu = sphere()
    tree = nk.OcTree(c, c, nodeCapacity=60, nearest=1, finePoints=f, NN=NN)
    fmm = nk.KIFMM(tree, [eps, mu], GMRES=1, format=fmt)
    # GMRES to 1e-8: below ~1e-9 the explicit residual of the FP64 FMM (exact
    # LU check-to-equivalent inverses) stops falling
    R = nk.Gen_Resistance(fmm, tol=1e-8, maxIter=500)
    # dense FP64 resistance problem of the same discretization
    A = kernel(f, c, eps, mu) @ sp.kron(NN, sp.identity(3)).toarray()
    Rd = np.zeros((6, 6))
    for j in range(6):
        vel, mom = np.zeros(3), np.zeros(3)
        (vel if j < 3 else mom)[j % 3] = 1.0
        fr = np.linalg.solve(A, velocityModes(c, vel, mom).ravel()).reshape(-1, 3)
        Rd[:3, j], Rd[3:, j] = force_moment(fr, c, NN, f)
    assert np.linalg.norm(R - Rd) <= 1e-4 * np.linalg.norm(Rd), np.linalg.norm(R - Rd) / np.linalg.norm(Rd)
    # the unit sphere's drag and rotational resistance (6 pi mu a, 8 pi mu a^3) to discretization error
    assert abs(R[0, 0] / (6 * np.pi) - 1) < 2e-2 and abs(R[5, 5] / (8 * np.pi) - 1) < 2e-2
    # the same FMM operator in mobility form: R = inverse of the 6 x 6 mobility matrix
    Mob, its = Body(c, f, [eps, mu], 60, "fp64").solve_modes(1e-8, 500)
    assert np.linalg.norm(R @ Mob - np.eye(6)) <= 1e-5
