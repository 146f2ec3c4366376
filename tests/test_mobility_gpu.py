"""GPU mobility solve of one rigid sphere (NEAREST, p=6, eps=0.01, 488 force points)
against the dense FP64 regularized-Stokeslet system, and the known answers
U = F/(6 pi mu a), Omega = M/(8 pi mu a^3)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN
from oracle import mobility as om

pytestmark = pytest.mark.gpu


def sphere_body(F, M):
    g = np.load(os.path.join(GOLDEN, "sphere10_40.npz"))
    NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
    c, f = g["coarse"], g["fine"]
    return c, f, NN, F, M


def run_problem(F, M, precon, precision="fp64", refine=None, tol=1e-8):
    c, f, NN, F, M = sphere_body(F, M)
    sw = nk.Swimmers()
    sw.addSwimmer(c, f, NN, [0, 0, 0], [1, 0, 0, 0, 1, 0], np.zeros_like(c), F, M)
    out, info = nk.mobilityProblem(sw, None, 0.0, np.array([0, 0, 0, 1, 0, 0, 0, 1, 0.0]), [0.01, 1.0],
                                   {"nodeCapacity": 60, "nearest": 1}, tol=tol, maxIter=300,
                                   PreconSettings=[1e-6, 100] if precon else None, precision=precision,
                                   return_info=True, refine=refine)
    body = om.Body(c, f, NN, [0, 0, 0], [1, 0, 0, 0, 1, 0], np.zeros_like(c), F, M)
    asm = om.assemble([body])
    xd = np.linalg.solve(om.dense_mobility_matrix(asm, 0.01, 1.0, True), om.mobility_rhs(asm))
    return out, info, xd


@pytest.mark.parametrize("precon", [False, True])
def test_translation_and_rotation(precon):
    out, info, xd = run_problem([1, 0, 0], [0, 0, 0], precon)
    assert info["flag"] == 0
    U = out[0:3]
    assert abs(U[0] - xd[-6]) / abs(xd[-6]) < 1e-5
    assert abs(U[0] * 6 * np.pi - 1) < 1e-2
    out, info, xd = run_problem([0, 0, 0], [0, 0, 1], precon)
    Om = np.cross([1, 0, 0], out[3:6])  # out(4:6) = Om x b1 with b1 = e_x
    assert info["flag"] == 0
    assert abs(out[3:6][1] - xd[-1]) / abs(xd[-1]) < 1e-5  # (Om x e_x)_y = Om_z
    assert abs(xd[-1] * 8 * np.pi - 1) < 2e-2
    del Om


def test_precon_reduces_iterations():
    # at tol 1e-6, well above the ~1e-9 rounding floor of the FP64 FMM, where
    # iteration counts near tol 1e-8 vary from run to run
    _, a, _ = run_problem([1, 0, 0], [0, 0, 1], False, tol=1e-6)
    _, b, _ = run_problem([1, 0, 0], [0, 0, 1], True, tol=1e-6)
    assert b["iters"] <= a["iters"]


def test_mobility_matvec_vs_dense():
    c, f, NN, _, _ = sphere_body(None, None)
    sw = nk.Swimmers()
    sw.addSwimmer(c, f, NN, [0.1, -0.2, 0.3], [0, 1, 0, -1, 0, 0], np.zeros_like(c), [0, 0, 0], [0, 0, 0])
    sw.genTree(nodeCapacity=60, nearest=1)
    sw.genKIFMM([0.01, 1.0], GMRES=1, format=2)
    mob = sw.mobility()
    body = om.Body(c, f, NN, [0.1, -0.2, 0.3], [0, 1, 0, -1, 0, 0], np.zeros_like(c), [0, 0, 0], [0, 0, 0])
    A = om.dense_mobility_matrix(om.assemble([body]), 0.01, 1.0, True)
    x = np.random.default_rng(4).standard_normal(A.shape[0])
    y = mob.apply(x)
    assert np.linalg.norm(y - A @ x) / np.linalg.norm(A @ x) < 1e-4
    # rigid rows are exact (no FMM involved)
    assert np.allclose(y[-6:], (A @ x)[-6:], rtol=1e-12, atol=1e-12)


def test_fmm_gmres_resistance_sphere():
    """gmres(@(x) fmm.computeVel(x), vel, [], 1e-8, 200): drag of a translating sphere."""
    c, f, NN, _, _ = sphere_body(None, None)
    t = nk.OcTree(c, c, nodeCapacity=60, nearest=1, finePoints=f, NN=NN)
    fmm = nk.KIFMM(t, [0.01, 1.0], GMRES=1, format=1)
    x, flag, relres, it = fmm.gmres(np.tile([1.0, 0, 0], len(c)), tol=1e-8, maxit=200)
    assert flag == 0 and relres <= 1e-8
    F = (NN @ x.reshape(-1, 3)).sum(0)
    assert abs(F[0] / (6 * np.pi) - 1) < 5e-3


@pytest.mark.parametrize("precon", [False, True])
def test_mixed_refined_solve_matches_dense(precon):
    """Mixed-precision GMRES with FP64 iterative refinement reaches the FP64
    operator's solution: rigid velocities within 1e-4 of the dense FP64 solve."""
    out, info, xd = run_problem([1, 0, 0], [0, 0, 1], precon, precision="mixed")
    assert info["flag"] == 0 and info["relres"] <= 1e-8
    U = out[0:3]
    Om_z = out[3:6][1]
    assert abs(U[0] - xd[-6]) / abs(xd[-6]) < 1e-4
    assert abs(Om_z - xd[-1]) / abs(xd[-1]) < 1e-4
    ref, _, _ = run_problem([1, 0, 0], [0, 0, 1], precon, precision="fp64")
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replayed_matvec_is_bitwise_the_launches(precision):
    """The mobility matvec replayed from a CUDA graph equals the kernel-by-
    kernel launches bit for bit, and a graph captured before set_eps is not
    reused after it (the operators changed)."""
    c, f, NN, F, M = sphere_body([1, 0, 0], [0, 0, 1])
    sw = nk.Swimmers()
    sw.addSwimmer(c, f, NN, [0, 0, 0], [1, 0, 0, 0, 1, 0], np.zeros_like(c), F, M)
    sw.genTree(nodeCapacity=60, nearest=1)
    sw.genKIFMM([0.01, 1.0], GMRES=1, format=2, precision=precision)
    mob = sw.mobility()
    x = np.random.default_rng(3).standard_normal(mob.n)
    mob.use_graphs(False)
    a = mob.apply(x)
    mob.use_graphs(True)
    b = mob.apply(x)   # captures
    c2 = mob.apply(x)  # replays
    assert np.array_equal(a, b) and np.array_equal(a, c2)
    sw.FMM.setEps(0.02)
    d = mob.apply(x)   # captured again
    mob.use_graphs(False)
    e = mob.apply(x)
    assert np.array_equal(d, e) and not np.array_equal(d, a)


def test_gravity_forcing_vs_dense():
    """mobilityProblemGravity.m: a sphere with its centre of mass offset along
    its axis b3, under gravity G: F = G, M = -4/3 pi offset (b3 x G); rigid
    velocities against the dense FP64 system with the same forcing."""
    c, f, NN, _, _ = sphere_body([0, 0, 0], [0, 0, 0])
    G, offset = np.array([0.3, 0.0, -1.0]), 0.2
    b = [1, 0, 0, 0, 1, 0]  # b3 = e_z
    sw = nk.Swimmers()
    sw.addSwimmer(c, f, NN, [0, 0, 0], b, np.zeros_like(c), [0, 0, 0], [0, 0, 0])
    out = nk.mobilityProblemGravity(sw, None, 0.0, np.array([0, 0, 0] + b, float), [0.01, 1.0],
                                    {"nodeCapacity": 60, "nearest": 1}, tol=1e-8, maxIter=300,
                                    gravPar=list(G) + [offset])
    M = -4.0 / 3.0 * np.pi * offset * np.cross([0, 0, 1.0], G)
    assert np.allclose(sw.F[0], G) and np.allclose(sw.Moment[0], M)
    body = om.Body(c, f, NN, [0, 0, 0], b, np.zeros_like(c), G, M)
    asm = om.assemble([body])
    xd = np.linalg.solve(om.dense_mobility_matrix(asm, 0.01, 1.0, True), om.mobility_rhs(asm))
    U, Om = xd[-6:-3], xd[-3:]
    ref = np.concatenate([U, np.cross(Om, [1, 0, 0]), np.cross(Om, [0, 1, 0])])
    assert np.linalg.norm(out - ref) <= 1e-5 * np.linalg.norm(ref)
    # it sinks at about G / (6 pi) and turns its heavy side down
    assert abs(out[2] * 6 * np.pi / G[2] - 1) < 1e-2 and abs(Om[1]) > 0


def test_initial_guess_and_hegedus_warm_start():
    """The solution at eps = 0.02, scaled by the Hegedus trick, as the initial
    guess of the eps = 0.01 solve (Data Generation/preconditioningInitalGuess.m):
    the same solution as a cold start, in no more iterations."""
    c, f, NN, F, M = sphere_body([1, 0, 0], [0, 0, 1])

    def mob_at(eps):
        sw = nk.Swimmers()
        sw.addSwimmer(c, f, NN, [0, 0, 0], [1, 0, 0, 0, 1, 0], np.zeros_like(c), F, M)
        sw.genTree(nodeCapacity=60, nearest=1)
        sw.genKIFMM([eps, 1.0], GMRES=1, format=2)
        return sw.mobility(), nk.mobilityRHS(sw)

    m2, b2 = mob_at(0.02)
    xp, flag, _, _ = m2.solve(b2, tol=1e-8, maxIter=300)
    assert flag == 0
    m1, b1 = mob_at(0.01)
    cold, flag_c, res_c, it_c = m1.solve(b1, tol=1e-8, maxIter=300)
    x0 = nk.hegedus(m1.apply, b1, xp)
    warm, flag_w, res_w, it_w = m1.solve(b1, tol=1e-8, maxIter=300, x0=x0)
    assert flag_c == 0 and flag_w == 0 and res_w <= 1e-8
    assert np.linalg.norm(m1.apply(warm) - b1) <= 2e-8 * np.linalg.norm(b1)
    # the rigid velocities agree to the solves' accuracy (the force densities of the
    # first-kind system less so)
    assert np.linalg.norm(warm[-6:] - cold[-6:]) <= 1e-6 * np.linalg.norm(cold[-6:])
    assert it_w <= it_c
