"""The block preconditioner of Mobility/MobilityPrecon.m:17-39 (nnk_mob_precon)
against its oracle restatement (oracle/mobility.py: mobility_precon, the
per-node-LU computeVelSparse and the per-leaf reducedSolve of the oracle
KIFMM on the same tree), on the rigid sphere and on two squirmers above a
wall (reduced size).  FP64: <= 1e-6 relative; mixed precision (Tikhonov
check-to-equivalent operators, FP32 pairs): <= 1e-3, the preconditioner only
steers GMRES."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN
from nnkifmm.workloads import two_squirmers_wall
from oracle import mobility as om
from oracle.kifmm import KIFMM as OKIFMM
from oracle.octree import OcTree as OTree

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def sphere_case():
    g = np.load(os.path.join(GOLDEN, "sphere10_40.npz"))
    NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
    c, f = g["coarse"], g["fine"]
    bodies = [om.Body(c, f, NN, [0.1, -0.2, 0.3], [0, 1, 0, -1, 0, 0], np.zeros_like(c), [0, 0, 0], [0, 0, 0])]

    def make(precision):
        sw = nk.Swimmers()
        sw.addSwimmer(c, f, NN, [0.1, -0.2, 0.3], [0, 1, 0, -1, 0, 0], np.zeros_like(c), [0, 0, 0], [0, 0, 0])
        sw.genTree(nodeCapacity=60, nearest=1)
        sw.genKIFMM([0.01, 1.0], GMRES=1, format=2, precision=precision)
        return sw
    return make, om.assemble(bodies), 0.01, 60


def squirmer_case():
    c = two_squirmers_wall(edge_force=6, edge_quad=12, wall_n=24, spacing=0.15)
    NN = nk.nearestMatrix(c["body"], c["fine"], builder="host")
    W = c["wall"]
    bodies = [om.Body(c["body"], c["fine"], NN, list(x0), [1, 0, 0, 0, 1, 0], c["slip"], [0, 0, 0], [0, 0, 0])
              for x0 in c["centres"]]

    def make(precision):
        sw = nk.Swimmers()
        for x0 in c["centres"]:
            sw.addSwimmer(c["body"], c["fine"], NN, list(x0), [1, 0, 0, 0, 1, 0], c["slip"], [0, 0, 0], [0, 0, 0])
        sw.updateBnd(W, W, sp.identity(len(W), format="csr"), np.zeros_like(W))
        sw.genTree(nodeCapacity=60, nearest=1)
        sw.genKIFMM([0.02, 1.0], GMRES=1, format=2, precision=precision)
        return sw
    asm = om.assemble(bodies, bnd_points=W, bnd_fine=W, bnd_NN=sp.identity(len(W), format="csr"),
                      bnd_vel=np.zeros_like(W))
    return make, asm, 0.02, 60


@pytest.mark.parametrize("case", ["sphere", "squirmers_wall"])
def test_precon_matches_oracle(case):
    make, asm, eps, cap = sphere_case() if case == "sphere" else squirmer_case()
    tree = OTree(asm["points"], asm["points"], node_capacity=cap, nearest=1, fine_points=asm["fine"], NN=asm["NN"])
    ofmm = OKIFMM(tree, eps, 1.0, gmres=1, fmt=2)
    rng = np.random.default_rng(11)
    n = 3 * len(asm["points"]) + 6 * asm["nb"]
    for precision, tol in [("fp64", 1e-6), ("mixed", 1e-3)]:
        mob = make(precision).mobility()
        assert mob.n == n
        for k in range(2):
            x = rng.standard_normal(n)
            if k == 1:
                x[:-6 * asm["nb"]] = 0.0  # the rigid-mode path alone (computeVelSparse branch)
            ref = om.mobility_precon(x, asm, ofmm)
            y = mob.precon(x)
            e = rel(y, ref)
            print(case, precision, k, "precon vs oracle", e)
            assert e <= tol
