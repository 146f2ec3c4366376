"""The host side of the Swimmers mirror (no GPU): the rotated and translated
points, fine points, block NN matrix, slip velocities and the right-hand side
of mobilityProblem.m:37-46 equal the oracle's assembly of the same bodies and
boundary (Classes/Swimmers.m:150-340), and updateSwimmmer /
updateSwimmmerRHS change what Swimmers.m:361-385 change."""
import numpy as np
import scipy.sparse as sp

import nnkifmm as nk
from oracle import mobility as om
from oracle.geometry import random_rotation, sphere
from oracle.nearest import nearest_matrix


def _bodies(rng, nb):
    out = []
    for k in range(nb):
        c = sphere(0.3 + 0.1 * k, [0, 0, 0], 5 + k)
        f = sphere(0.3 + 0.1 * k, [0, 0, 0], 9 + k)
        R = random_rotation(rng)
        out.append(dict(points=c, fine=f, NN=nearest_matrix(c, f), x0=rng.uniform(-2, 2, 3),
                        b=np.concatenate([R[:, 0], R[:, 1]]), vel=rng.standard_normal(c.shape),
                        F=rng.standard_normal(3), M=rng.standard_normal(3)))
    return out


def _pair(rng, nb=3, boundary=True):
    bodies = _bodies(rng, nb)
    sw = nk.Swimmers()
    for b in bodies:
        sw.addSwimmer(b["points"], b["fine"], b["NN"], b["x0"], b["b"], b["vel"], b["F"], b["M"])
    obodies = [om.Body(b["points"], b["fine"], b["NN"], b["x0"], b["b"], b["vel"], b["F"], b["M"]) for b in bodies]
    if not boundary:
        return sw, om.assemble(obodies)
    W = np.stack(np.meshgrid(np.linspace(-3, 3, 12), np.linspace(-3, 3, 12), [-2.5], indexing="ij"), -1).reshape(-1, 3)
    WV = rng.standard_normal(W.shape)
    sw.updateBnd(W, W, sp.identity(len(W), format="csr"), WV)
    return sw, om.assemble(obodies, W, W, sp.identity(len(W), format="csr"), WV)


def test_assembly_matches_the_oracle():
    sw, asm = _pair(np.random.default_rng(41))
    P, Fp, NN = sw.getSwimmerBnd()
    assert np.array_equal(P, asm["points"]) and np.array_equal(Fp, asm["fine"])
    assert (NN != asm["NN"]).nnz == 0 and NN.shape == asm["NN"].shape
    assert np.array_equal(sw.getVelocities(), asm["vel"])
    _, _, _, rel, frel = sw.getSwimmers()
    assert np.array_equal(rel, asm["rel"]) and np.array_equal(frel, asm["frel"])
    sizes, fsizes = sw.getSwimmerSizes()
    assert np.array_equal(np.concatenate([[0], np.cumsum(sizes)]), asm["bstart"])
    assert np.array_equal(np.concatenate([[0], np.cumsum(fsizes)]), asm["fstart"])


def test_right_hand_side_with_background_flow():
    """The background flow is subtracted on the swimmer rows only."""
    sw, asm = _pair(np.random.default_rng(42))

    def shear(t, x):
        v = np.zeros_like(x)
        v[:, 0] = 2.0 * x[:, 2]
        return v
    b = nk.mobilityRHS(sw, shear, 0.0)
    ref = om.mobility_rhs(asm, lambda x: shear(0.0, x))
    assert b.shape == ref.shape and np.array_equal(b, ref)
    assert np.array_equal(nk.mobilityRHS(sw), om.mobility_rhs(asm))


def test_update_swimmer_and_gravity_forcing():
    rng = np.random.default_rng(43)
    sw, _ = _pair(rng, nb=2, boundary=False)
    R = random_rotation(rng)
    sw.updateSwimmmer(2, [0.5, -0.5, 1.0], np.concatenate([R[:, 0], R[:, 1]]))
    pts = sw.getSwimmers()[0]
    n0 = sw.getSwimmerSizes()[0][0]
    assert np.allclose(pts[n0:], (R @ sw.Geometries[1].T).T + [0.5, -0.5, 1.0], rtol=0, atol=1e-15)
    G, off = np.array([0.0, 0.0, -1.0]), 0.2
    sw.updateSwimmmerRHS(2, G, off)
    F, M = sw.getForceMoment()
    assert np.array_equal(F[3:], G)
    assert np.allclose(M[3:], -4.0 / 3.0 * np.pi * off * np.cross(R[:, 2], G), rtol=0, atol=1e-15)
