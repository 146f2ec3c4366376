"""The differentiation configuration at its stated size: a prolate spheroid
(a = 1, c = 3) with about 50k force and 200k quadrature points, eps = 0.005,
free space, a unit force in x; loss ||[U; Om] - U*||^2 with U* ~ N(0,1).
The gradient of rigid_velocity (adjoint GMRES, the kernel's position
derivative through the FMM's leaf stages, the rigid-body blocks) against
central finite differences of the FP64 solve itself along 32 random
directions of the force and quadrature points, for the FP64 and the
mixed-precision solves, at the configuration's step h = 1e-6 and at 1e-5.

What the directions leave still (displacements are below h/10 per point):
* the gradient holds the nearest map fixed, so the quadrature points whose
  two nearest force points are within h of a tie, and those force points
  (the points are jittered, so there are few: 5,192 of the 200k within
  1e-5, the larger step);
* the gradient is that of the FMM operator on its tree, so the points that
  set the root cube and the force points within h of a box face: otherwise
  the difference also sees the FMM's approximation error change with the
  box geometry (9% on these directions).
A direction along which some nearest force point still changes is drawn
again.  The solves run on FP64 Tikhonov operators (rounding ~1e-11 instead
of the exact inverse's ~1e-9) to a relative residual of 1e-11, about the
floor GMRES reaches here (3.7e-12 after 1000 iterations); their error,
amplified by the system's condition number and divided by 2h, is the noise
of the differences: 0.5% at h = 1e-6, ten times less at h = 1e-5, where the
bound applies.  Takes about four minutes on a B200."""
import numpy as np
import pytest
import torch
from scipy.spatial import cKDTree

import nnkifmm as nk
from nnkifmm.autograd import rigid_velocity
from nnkifmm.workloads import _spacing_for_count, prolate_spheroid

pytestmark = pytest.mark.gpu


def test_gradient_against_32_fd_directions_at_50k():
    rng = np.random.default_rng(20261210)
    h0 = _spacing_for_count(1.0, 3.0, 50_000)
    X0 = prolate_spheroid(1.0, 3.0, h0)
    Y0 = prolate_spheroid(1.0, 3.0, h0 / 2)
    X0 = X0 + 1e-3 * h0 * rng.standard_normal(X0.shape)
    Y0 = Y0 + 1e-3 * h0 * rng.standard_normal(Y0.shape)
    eps, F, M = 0.005, np.array([1.0, 0.0, 0.0]), np.zeros(3)
    Us = rng.standard_normal(6)
    NN = nk.nearestMatrix(X0, Y0)
    opts = dict(cap=64, tol=1e-11, maxIter=1000, reg=1e-5)

    def loss(X, Y):
        U = rigid_velocity(torch.tensor(X), torch.tensor(Y), eps, F, M, precision="fp64", **opts)
        return float(((U - torch.tensor(Us)) ** 2).sum())

    grads = {}
    for prec, tol in [("fp64", 1e-11), ("mixed", 1e-8)]:
        X = torch.tensor(X0, requires_grad=True)
        Y = torch.tensor(Y0, requires_grad=True)
        U = rigid_velocity(X, Y, eps, F, M, precision=prec, **dict(opts, tol=tol))
        ((U - torch.tensor(Us)) ** 2).sum().backward()
        grads[prec] = (X.grad.numpy().copy(), Y.grad.numpy().copy())
    steps = (1e-6, 1e-5)
    lim = max(steps)  # ties and faces closer than the largest step stay still
    d2, i2 = cKDTree(X0).query(Y0, k=2)
    tied = d2[:, 1] - d2[:, 0] < lim
    still_x = np.zeros(len(X0), bool)
    still_x[i2[tied].ravel()] = True
    for P, still in ((X0, still_x), (Y0, tied)):
        for ax in range(3):
            still |= (P[:, ax] <= P[:, ax].min() + 1e-12) | (P[:, ax] >= P[:, ax].max() - 1e-12)
    T = nk.OcTree(X0, X0, nodeCapacity=opts["cap"], nearest=1, finePoints=Y0, NN=NN)
    root = np.asarray(T.nodeCorners)[0]  # node 0 is the root: [lo hi]
    cell = (root[3] - root[0]) / 2.0 ** int(np.asarray(T.nodeLevel).max())
    u = (X0 - root[:3]) / cell
    still_x |= (np.abs(u - np.rint(u)) * cell < lim).any(axis=1)
    del T
    fd, an = {h: [] for h in steps}, {p: [] for p in grads}
    tries = 0
    while len(an["fp64"]) < 32:
        tries += 1
        assert tries <= 200, "too few directions keep the nearest map"
        dX = rng.standard_normal(X0.shape)
        dY = rng.standard_normal(Y0.shape)
        dX[still_x] = 0.0
        dY[tied] = 0.0
        nrm = np.sqrt((dX * dX).sum() + (dY * dY).sum())
        dX, dY = dX / nrm, dY / nrm
        if any((nk.nearestMatrix(X0 + s * lim * dX, Y0 + s * lim * dY) != NN).nnz for s in (-1, 1)):
            continue
        for h in steps:
            fd[h].append((loss(X0 + h * dX, Y0 + h * dY) - loss(X0 - h * dX, Y0 - h * dY)) / (2 * h))
        for p, (gX, gY) in grads.items():
            an[p].append(float((gX * dX).sum() + (gY * dY).sum()))
    errs = {(p, h): float(np.linalg.norm(np.array(an[p]) - np.array(fd[h])) / np.linalg.norm(fd[h]))
            for p in an for h in steps}
    print("points", len(X0), len(Y0), "still", int(tied.sum()), int(still_x.sum()), "directions drawn", tries,
          "directional-derivative error vs FD over 32 directions (precision, h):", errs)
    assert errs[("fp64", 1e-5)] <= 1e-3
    assert errs[("mixed", 1e-5)] <= 1e-2
    assert errs[("fp64", 1e-6)] <= 2e-2
