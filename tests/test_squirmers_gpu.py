"""Two squirmers above a wall (the squirmer configuration at reduced size):
B1/B2 tangential slip, force- and torque-free bodies, a wall boundary with
NN = I and zero velocity, the block preconditioner of MobilityPrecon.m, FP64
and mixed precision with FP64 refinement, and Richardson extrapolation over
eps.  Checked against the dense FP64 mobility system of the oracle."""
import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from nnkifmm.workloads import two_squirmers_wall
from oracle import mobility as om

pytestmark = pytest.mark.gpu

MU = 1.0


@pytest.fixture(scope="module")
def case():
    return two_squirmers_wall(edge_force=6, edge_quad=12, wall_n=24, spacing=0.15)


def swimmers(c):
    sw = nk.Swimmers()
    NN = nk.nearestMatrix(c["body"], c["fine"])
    for x0 in c["centres"]:
        sw.addSwimmer(c["body"], c["fine"], NN, list(x0), [1, 0, 0, 0, 1, 0], c["slip"], [0, 0, 0], [0, 0, 0])
    W = c["wall"]
    sw.updateBnd(W, W, sp.identity(len(W), format="csr"), np.zeros_like(W))
    return sw, NN


def conditions(c):
    return np.concatenate([np.concatenate([x0, [1, 0, 0], [0, 1, 0]]) for x0 in c["centres"]])


def dense(c, NN, eps):
    bodies = [om.Body(c["body"], c["fine"], NN, list(x0), [1, 0, 0, 0, 1, 0], c["slip"], [0, 0, 0], [0, 0, 0])
              for x0 in c["centres"]]
    W = c["wall"]
    asm = om.assemble(bodies, bnd_points=W, bnd_fine=W, bnd_NN=sp.identity(len(W), format="csr"),
                      bnd_vel=np.zeros_like(W))
    x = np.linalg.solve(om.dense_mobility_matrix(asm, eps, MU, True), om.mobility_rhs(asm))
    return om.rigid_output(asm, x, bodies)


def gpu(c, eps, precision, precon=True):
    sw, NN = swimmers(c)
    out, info = nk.mobilityProblem(sw, None, 0.0, conditions(c), [eps, MU], {"nodeCapacity": 60, "nearest": 1},
                                   tol=1e-8, maxIter=500, PreconSettings=[1e-6, 100] if precon else None,
                                   precision=precision, return_info=True)
    return out, info, NN


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-5), ("mixed", 1e-4)])
def test_two_squirmers_wall_vs_dense(case, precision, tol):
    out, info, NN = gpu(case, 0.02, precision)
    assert info["flag"] == 0
    ref = dense(case, NN, 0.02)
    assert np.linalg.norm(out - ref) <= tol * np.linalg.norm(ref), (np.linalg.norm(out - ref) / np.linalg.norm(ref))
    # the squirmers swim: nonzero rigid velocity along their axes
    assert abs(out[2]) > 1e-3 and abs(out[11]) > 1e-3


def test_preconditioner_keeps_the_solution(case):
    a, ia, _ = gpu(case, 0.02, "fp64", precon=False)
    b, ib, _ = gpu(case, 0.02, "fp64", precon=True)
    assert ia["flag"] == 0 and ib["flag"] == 0
    assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(a)


def test_richardson_over_eps(case):
    """Extrapolated rigid velocities from eps = 0.02 and 0.01 (mixed with
    refinement) against the same extrapolation of the dense solutions."""
    eps = (0.02, 0.01)
    outs, refs = [], []
    for e in eps:
        o, info, NN = gpu(case, e, "mixed")
        assert info["flag"] == 0
        outs.append(o)
        refs.append(dense(case, NN, e))
    r_gpu = nk.richardson(outs, eps)
    r_ref = nk.richardson(refs, eps)
    assert np.linalg.norm(r_gpu - r_ref) <= 2e-4 * np.linalg.norm(r_ref)
    # the formula removes an O(eps) error exactly
    lin = [np.array([1.0, 2.0]) + e * np.array([3.0, -1.0]) for e in eps]
    assert np.allclose(nk.richardson(lin, eps), [1.0, 2.0])
