"""The FP64 oracle against the reference's known answers and self-consistency.

The reference ships no golden vectors; its one built-in known answer is the
Stokes drag of the unit sphere, [6*pi; 0; 0]
(Data Generation/DirectMethodComparison.m:34, Benchmarkresistance.m:12,35).
"""
import os

import numpy as np
import pytest

from oracle import mobility as om
from oracle.geometry import sphere, prolate_spheroid, velocity_modes, wall_tri
from oracle.gmres import gmres
from oracle.kernel import apply_kernel, kernel
from oracle.mlab import linspace
from oracle.nearest import nearest_matrix
from oracle.octree import OcTree, MaxDepthError
from oracle.surfaces import downsurf, surface_count, upsurf


def test_matlab_linspace_endpoints_and_formula():
    y = linspace(-1.0, 1.0, 7)
    assert y[0] == -1.0 and y[-1] == 1.0
    k = np.arange(7.0)
    assert np.array_equal(y[1:-1], (-1.0 + (k * 2.0) / 6)[1:-1])


def test_sphere_counts():
    # n^3 - (n-2)^3 points (Geometries/Sphere.m)
    assert sphere(1.0, [0, 0, 0], 10).shape == (488, 3)
    assert sphere(1.0, [0, 0, 0], 40).shape == (9128, 3)
    p = sphere(2.0, [1, 2, 3], 6)
    assert np.allclose(np.linalg.norm(p - [1, 2, 3], axis=1), 2.0)


def test_surfaces_counts_and_order():
    assert surface_count(6, 1) == 152 and surface_count(4, 1) == 56
    c = np.array([0.0, 0, 0, 1, 1, 1])
    u = upsurf(c)
    d = downsurf(c)
    assert u.shape == (152, 3) and d.shape == (152, 3)
    # column-major meshgrid order: y runs fastest, then x, then z
    assert np.array_equal(u[0], [0, 0, 0]) and np.array_equal(u[1], [0, 0.2, 0])
    assert d.min() == -1.0 and d.max() == 2.0


def test_kernel_symmetry_and_blocks():
    rng = np.random.default_rng(0)
    x, y = rng.random((5, 3)), rng.random((4, 3))
    S = kernel(x, y, 0.1, 1.3)
    assert np.allclose(S, kernel(y, x, 0.1, 1.3).T, rtol=0, atol=1e-14)
    f = rng.standard_normal((5, 3))
    assert np.allclose((S @ f.ravel()).reshape(-1, 3), apply_kernel(x, y, f, 0.1, 1.3), rtol=1e-13)


def test_sphere_drag_known_answer():
    """F = 6 pi mu a U for a translating unit sphere (DirectMethodComparison.m:34)."""
    c = sphere(1.0, [0, 0, 0], 10)
    f = sphere(1.0, [0, 0, 0], 40)
    NN = nearest_matrix(c, f)
    A = kernel(f, c, 0.01, 1.0) @ np.kron(NN.toarray(), np.eye(3))
    x = np.linalg.solve(A, np.tile([1.0, 0, 0], len(c)))
    F = (NN @ x.reshape(-1, 3)).sum(0)
    assert abs(F[0] - 6 * np.pi) / (6 * np.pi) < 5e-3
    assert abs(F[1]) < 1e-10 and abs(F[2]) < 1e-10


def test_mobility_sphere_known_answers():
    """U = F/(6 pi mu a), Omega = M/(8 pi mu a^3) for the rigid sphere of 488 force points."""
    c = sphere(1.0, [0, 0, 0], 10)
    f = sphere(1.0, [0, 0, 0], 40)
    NN = nearest_matrix(c, f)
    body = om.Body(c, f, NN, [0, 0, 0], [1, 0, 0, 0, 1, 0], np.zeros_like(c), [1, 0, 0], [0, 0, 1])
    asm = om.assemble([body])
    M = om.dense_mobility_matrix(asm, 0.01, 1.0, True)
    x = np.linalg.solve(M, om.mobility_rhs(asm))
    assert abs(x[-6] * 6 * np.pi - 1) < 1e-2
    assert abs(x[-1] * 8 * np.pi - 1) < 2e-2


def test_nearest_ties_share_weight():
    g = np.array([[i, j, k] for i in range(3) for j in range(3) for k in range(3)], float)
    NN = nearest_matrix(g, np.array([[0.5, 0.5, 0.5], [0.1, 0, 0]]))
    assert NN.getnnz(axis=1).tolist() == [8, 1]
    assert np.allclose(NN.sum(axis=1), 1.0)
    assert np.allclose(NN[0].data, 1 / 8)


def test_octree_capacity_and_dfs_ids():
    rng = np.random.default_rng(3)
    x = rng.random((500, 3))
    t = OcTree(x, x, node_capacity=20, build_lists=False)
    leaves = np.nonzero(t.children[1:, 0] == 0)[0] + 1
    counts = np.bincount(t.point_index, minlength=t.node_count + 1)
    assert counts[leaves].max() <= 20
    # children of a node are a consecutive block of 8 ids, appended in DFS order
    for i in range(1, t.node_count + 1):
        ch = t.children[i]
        if ch[0]:
            assert np.array_equal(ch, np.arange(ch[0], ch[0] + 8))
            assert (t.parent[ch] == i).all()


def test_octree_max_depth_error():
    x = np.array([[0, 0, 0], [1e-9, 0, 0], [1, 1, 1]], float)
    with pytest.raises(MaxDepthError):
        OcTree(x, x, node_capacity=1, max_depth=8)


def test_oracle_gmres_matches_dense_solve():
    rng = np.random.default_rng(1)
    A = np.eye(40) + 0.1 * rng.standard_normal((40, 40))
    b = rng.standard_normal(40)
    x, flag, relres, it, _ = gmres(lambda v: A @ v, b, None, 1e-12, 40)
    assert flag == 0 and relres <= 1e-12
    assert np.allclose(x, np.linalg.solve(A, b), rtol=1e-9, atol=1e-10)


def test_geometry_generators():
    p = prolate_spheroid(0.5, 1.5, 0.2)
    assert np.allclose(p[:2], [[0, 0, 1.5], [0, 0, -1.5]])
    r = (p[:, 0] ** 2 + p[:, 1] ** 2) / 0.25 + p[:, 2] ** 2 / 2.25
    assert np.allclose(r, 1.0)
    w = wall_tri([0, 0, -1.5], [1.0, 1.0], 3, 0.05)
    assert np.allclose(w[:, 2], -1.5) and len(w) > 400
    v = velocity_modes(np.eye(3), [1, 0, 0], [0, 0, 1])
    assert np.allclose(v, [[1, 1, 0], [0, 0, 0], [1, 0, 0]])


def test_dense_gradient_matches_finite_differences():
    """The dense adjoint gradient (oracle/gradient.py) against central
    differences of the dense loss, on a small body."""
    from oracle import gradient as og
    from oracle.geometry import sphere as cube_sphere
    from oracle.nearest import nearest_matrix
    rng = np.random.default_rng(4)
    X = cube_sphere(1.0, (0, 0, 0), 4) * np.array([1.0, 0.8, 1.3])
    Y = cube_sphere(1.0, (0, 0, 0), 8) * np.array([1.0, 0.8, 1.3])
    NN = nearest_matrix(X, Y)
    eps, mu = 0.05, 1.0
    F, M, Us = rng.standard_normal(3), rng.standard_normal(3), rng.standard_normal(6)
    L, gX, gY, ge = og.gradient(X, Y, NN, eps, mu, F, M, Us)
    h = 1e-6
    for k in range(3):
        dX, dY = rng.standard_normal(X.shape), rng.standard_normal(Y.shape)
        lp = og.loss(X + h * dX, Y + h * dY, NN, eps, mu, F, M, Us)
        lm = og.loss(X - h * dX, Y - h * dY, NN, eps, mu, F, M, Us)
        fd = (lp - lm) / (2 * h)
        an = float((gX * dX).sum() + (gY * dY).sum())
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)
    lp = og.loss(X, Y, NN, eps + h, mu, F, M, Us)
    lm = og.loss(X, Y, NN, eps - h, mu, F, M, Us)
    assert abs((lp - lm) / (2 * h) - ge) <= 1e-6 * max(1.0, abs(ge))


def test_resistance_formulas_invert_the_dense_mobility_matrix():
    """The resistance problem (Rigid_Resistance.m / Gen_Resistance.m: impose
    U + Omega x X, solve S kron(NN, I3) f = u, sum forces and moments) with
    the dense FP64 operator gives the inverse of the dense 6 x 6 mobility
    matrix of the same discretization, and the point velocities follow
    velocityModes.m."""
    import scipy.sparse as sp
    from nnkifmm.resistance import force_moment, velocityModes
    from oracle import mobility as om
    from oracle.geometry import sphere, velocity_modes
    from oracle.kernel import kernel
    from oracle.nearest import nearest_matrix
    c, f = sphere(1.0, [0, 0, 0], 5), sphere(1.0, [0, 0, 0], 12)
    NN = sp.csr_matrix(nearest_matrix(c, f))
    eps, mu = 0.05, 1.0
    rng = np.random.default_rng(4)
    X = rng.random((7, 3))
    assert np.allclose(velocityModes(X, [1, 2, 3], [0.5, -1, 2]), velocity_modes(X, [1, 2, 3], [0.5, -1, 2]))
    A = kernel(f, c, eps, mu) @ sp.kron(NN, sp.identity(3)).toarray()
    R = np.zeros((6, 6))
    for j in range(6):
        vel, mom = np.zeros(3), np.zeros(3)
        (vel if j < 3 else mom)[j % 3] = 1.0
        fr = np.linalg.solve(A, velocityModes(c, vel, mom).ravel()).reshape(-1, 3)
        F, M = force_moment(fr, c, NN, f)
        R[:3, j], R[3:, j] = F, M
    Mob = np.zeros((6, 6))
    for j in range(6):
        F, M = np.zeros(3), np.zeros(3)
        (F if j < 3 else M)[j % 3] = 1.0
        body = om.Body(c, f, NN, [0, 0, 0], [1, 0, 0, 0, 1, 0], np.zeros_like(c), F, M)
        asm = om.assemble([body])
        Mob[:, j] = np.linalg.solve(om.dense_mobility_matrix(asm, eps, mu, True), om.mobility_rhs(asm))[-6:]
    assert np.linalg.norm(R @ Mob - np.eye(6)) <= 1e-8
    assert np.linalg.norm(R - R.T) <= 1e-6 * np.linalg.norm(R)  # the grand resistance matrix is symmetric


def test_hegedus_scale_minimises_the_residual():
    """x0 = scale * xp with scale = (b' A xp) / ||A xp||^2 minimises
    ||b - A x0|| over multiples of xp (Tests/HegadusTrickTest.m)."""
    from nnkifmm.mobility import hegedus
    rng = np.random.default_rng(6)
    A = rng.standard_normal((30, 30)) + 30 * np.eye(30)
    b, xp = rng.standard_normal(30), rng.standard_normal(30)
    x0 = hegedus(lambda v: A @ v, b, xp)
    r = lambda s: np.linalg.norm(b - A @ (s * xp))
    s0 = float(x0 @ xp / (xp @ xp))
    assert r(s0) <= min(r(s0 * 1.001), r(s0 * 0.999))


def test_parfor_matvec_matches_the_serial_oracle():
    """The reference arm's matvec (the reference's parfor loops over the nodes
    of a level on spawned worker processes, one BLAS thread each) gives the
    serial oracle's velocities on the NEAREST golden case."""
    import scipy.sparse as sp
    from threadpoolctl import threadpool_limits

    from conftest import GOLDEN
    from oracle.kifmm import KIFMM
    from oracle.octree import OcTree
    from oracle.parfor import ParforKIFMM
    g = np.load(os.path.join(GOLDEN, "adaptive_nearest_1200.npz"))
    NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
    tree = OcTree(g["coarse"], g["coarse"], node_capacity=int(g["cap"]), nearest=1, fine_points=g["fine"], NN=NN)
    fmm = ParforKIFMM(tree, float(g["eps"]), float(g["mu"]), 2)
    try:
        v = fmm.compute_vel(g["F"])
        v2 = fmm.compute_vel(2.0 * g["F"])
    finally:
        fmm.close()
    with threadpool_limits(1):
        ref = KIFMM(tree, float(g["eps"]), float(g["mu"])).compute_vel(g["F"])
    assert np.abs(v - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(v2 - 2.0 * ref).max() <= 1e-12 * np.abs(ref).max()  # state reset between calls
    # the fixture was made with multi-threaded BLAS: LU rounding, lifted by cond ~1e10
    assert np.abs(v - g["vel"]).max() <= 1e-7 * np.abs(ref).max()
