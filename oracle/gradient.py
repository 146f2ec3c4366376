"""Dense FP64 gradient of a rigid-velocity loss (test infrastructure only, see
oracle/__init__.py).

The reference has no gradients; this is the dense oracle for the adjoint
path.  For one free body with force points X (N x 3), quadrature points
Y (Q x 3) and the nearest-neighbour matrix NN (held fixed: it is piecewise
constant in the positions), the mobility system of mobilityProblem.m:37-58
    A z = b,  A = [S(Y -> X) kron(NN, I3)  BT; B  0],  z = [f; U; Om],
with S the regularized Stokeslet of Tools/kernel.m:23-47 and B, BT of
Mobility/genMatrixComponets.m:16-100 (BT on X - x0, B's torque arm
sum_q NN(q, n) (Y_q - x0)), and the loss L = ||[U; Om] - U*||^2, the
gradient is dL/dtheta = -lam^T (dA/dtheta) z with A^T lam = dL/dz, written
out with the kernel's derivatives:
    d/dt [w . K(t - s) g] = [2 (w.g) r + (r.g) w + (w.r) g] / D^{3/2}
                            - 3 [(w.g)(r^2 + 2 eps^2) + (w.r)(r.g)] r / D^{5/2}
    dK/deps = eps [(r^2 - 2 eps^2) I - 3 r r^T] / D^{5/2}
(r = t - s, D = r^2 + eps^2, both over 8 pi mu).
"""
import numpy as np
import scipy.sparse as sp

from . import mobility as om


def _pairs(X, Y):
    r = X[:, None, :] - Y[None, :, :]
    r2 = (r * r).sum(-1)
    return r, r2


def solve_system(X, Y, NN, eps, mu, F, M):
    """z = A^-1 b for one free body at x0 = 0, rest orientation, no slip."""
    body = om.Body(X, Y, sp.csr_matrix(NN), [0, 0, 0], [1, 0, 0, 0, 1, 0], np.zeros_like(X), F, M)
    asm = om.assemble([body])
    A = om.dense_mobility_matrix(asm, eps, mu, True)
    b = om.mobility_rhs(asm)
    return A, b, np.linalg.solve(A, b)


def loss(X, Y, NN, eps, mu, F, M, Ustar):
    _, _, z = solve_system(X, Y, NN, eps, mu, F, M)
    d = z[-6:] - Ustar
    return float(d @ d)


def gradient(X, Y, NN, eps, mu, F, M, Ustar):
    """(L, dL/dX (N x 3), dL/dY (Q x 3), dL/deps) of L = ||[U; Om] - U*||^2."""
    X = np.asarray(X, float)
    Y = np.asarray(Y, float)
    NN = sp.csr_matrix(NN)
    N = len(X)
    A, b, z = solve_system(X, Y, NN, eps, mu, F, M)
    d = z[-6:] - Ustar
    L = float(d @ d)
    gz = np.zeros_like(z)
    gz[-6:] = 2 * d
    lam = np.linalg.solve(A.T, gz)
    f = z[:3 * N].reshape(3, N).T      # blocked layout (mobilityProblem.m:45-46)
    lf = lam[:3 * N].reshape(3, N).T
    Om = z[3 * N + 3:3 * N + 6]
    lM = lam[3 * N + 3:3 * N + 6]
    g = NN @ f                         # forces on the quadrature points
    r, r2 = _pairs(X, Y)
    e2 = eps * eps
    D = r2 + e2
    c = 1.0 / (8 * np.pi * mu)
    inv3 = D ** -1.5 * c
    inv5 = D ** -2.5 * c
    wg = lf @ g.T                      # (N, Q): lam_n . g_q
    wr = np.einsum("nk,nqk->nq", lf, r)
    rg = np.einsum("nqk,qk->nq", r, g)
    a = 2 * wg * inv3 - 3 * (wg * (r2 + 2 * e2) + wr * rg) * inv5
    # d/dX_n of lam_n . K(X_n - Y_q) g_q, summed over q (and -, over n, for Y_q)
    term = a[..., None] * r + (rg * inv3)[..., None] * lf[:, None, :] + (wr * inv3)[..., None] * g[None, :, :]
    J = term.sum(1)
    H = -term.sum(0)
    gX = -(J + np.cross(Om, lf))
    torque = np.cross(f, lM)           # d/dY_q of lam_M . sum_n xm_n x f_n, per n
    gY = -(H + NN @ torque)
    dK = eps * ((r2 - 2 * e2) * wg - 3 * wr * rg) * inv5
    geps = -float(dK.sum())
    return L, gX, gY, geps
