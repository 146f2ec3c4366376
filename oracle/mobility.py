"""Rigid-body mobility problem (FP64, dense), restated from Classes/Swimmers.m,
Mobility/genMatrixComponets.m, Mobility/MobilityMatrixMulti.m,
Mobility/MobilityPrecon.m and Mobility/mobilityProblem.m.

Test infrastructure only (see oracle/__init__.py).  The dense system
(regularized-Stokeslet matrix times kron(NN,I3), plus the rigid-body rows)
is the FP64 oracle for the mobility solves.
"""
import numpy as np
import scipy.sparse as sp

from .kernel import kernel


def basis(b1, b2):
    """B = [b1 b2 b1xb2] (Swimmers.m:180-183)."""
    b1 = np.asarray(b1, float)
    b2 = np.asarray(b2, float)
    return np.stack([b1, b2, np.cross(b1, b2)], axis=1)


class Body:
    """One swimmer as stored by Swimmers.addSwimmer (Swimmers.m:109-120):
    body-frame points / fine points / NN, centre x0, basis (b1,b2), body-frame
    slip velocity at the points, total force F and moment M."""

    def __init__(self, points, fine, NN, x0, b1b2, vel, F, M):
        self.points = np.asarray(points, float)
        self.fine = None if fine is None else np.asarray(fine, float)
        self.NN = None if NN is None else sp.csr_matrix(NN)
        self.x0 = np.asarray(x0, float).ravel()
        b = np.asarray(b1b2, float).ravel()
        self.b1, self.b2 = b[0:3], b[3:6]
        self.vel = np.asarray(vel, float)
        self.F = np.asarray(F, float).ravel()
        self.M = np.asarray(M, float).ravel()


def assemble(bodies, bnd_points=None, bnd_fine=None, bnd_NN=None, bnd_vel=None):
    """getSwimmerBnd / getSwimmers / getVelocities (Swimmers.m:150-340):
    rotated+translated global arrays, rotated untranslated copies, block NN."""
    pts, fine, rel, frel, vel, nns = [], [], [], [], [], []
    bstart, fstart = [0], [0]
    for b in bodies:
        B = basis(b.b1, b.b2)
        r = (B @ b.points.T).T
        rel.append(r)
        pts.append(r + b.x0)
        vel.append((B @ b.vel.T).T)
        bstart.append(bstart[-1] + len(b.points))
        if b.fine is not None:
            fr = (B @ b.fine.T).T
            frel.append(fr)
            fine.append(fr + b.x0)
            nns.append(b.NN)
            fstart.append(fstart[-1] + len(b.fine))
    out = dict(nb=len(bodies), bstart=np.array(bstart), fstart=np.array(fstart))
    out["rel"] = np.concatenate(rel) if rel else np.zeros((0, 3))
    out["frel"] = np.concatenate(frel) if frel else np.zeros((0, 3))
    P = np.concatenate(pts) if pts else np.zeros((0, 3))
    Fp = np.concatenate(fine) if fine else np.zeros((0, 3))
    V = np.concatenate(vel) if vel else np.zeros((0, 3))
    NNs = list(nns)
    if bnd_points is not None and len(bnd_points):
        P = np.concatenate([P, bnd_points])
        V = np.concatenate([V, bnd_vel if bnd_vel is not None else np.zeros_like(bnd_points)])
        if bnd_fine is not None:
            Fp = np.concatenate([Fp, bnd_fine])
            NNs.append(sp.csr_matrix(bnd_NN))
    out["points"] = P
    out["fine"] = Fp
    out["NN"] = sp.block_diag(NNs, format="csr") if NNs else None
    out["vel"] = V
    out["Fsw"] = np.array([b.F for b in bodies])
    out["Msw"] = np.array([b.M for b in bodies])
    return out


def gen_matrix_components(asm, nearest):
    """[B, BT, A1, A2] of Mobility/genMatrixComponets.m:16-100, dense, for the
    blocked layouts [f_x f_y f_z] (3N) and [U_x U_y U_z Om_x Om_y Om_z] (6 nb)."""
    N = len(asm["points"])
    nb = asm["nb"]
    bs = asm["bstart"]
    rel = asm["rel"]
    Nsw = bs[-1]
    au = np.zeros((N, nb))
    for b in range(nb):
        au[bs[b]:bs[b + 1], b] = -1.0
    AU = np.kron(np.eye(3), au)
    xm = [np.zeros((N, nb)) for _ in range(3)]
    for b in range(nb):
        for d in range(3):
            xm[d][bs[b]:bs[b + 1], b] = rel[bs[b]:bs[b + 1], d]
    Z = np.zeros((N, nb))
    AOm = np.block([[Z, -xm[2], xm[1]], [xm[2], Z, -xm[0]], [-xm[1], xm[0], Z]])
    if nearest:
        Q = asm["fstart"][-1]
        NN = asm["NN"][:Q, :Nsw].toarray()
        colsum = NN.sum(axis=0)
        pm = asm["frel"][:Q].T @ NN  # (3, Nsw): sum_q NN(q,n) X_q
    else:
        colsum = np.ones(Nsw)
        pm = rel[:Nsw].T
    af = np.zeros((nb, N))
    x_m = [np.zeros((nb, N)) for _ in range(3)]
    for b in range(nb):
        af[b, bs[b]:bs[b + 1]] = colsum[bs[b]:bs[b + 1]]
        for d in range(3):
            x_m[d][b, bs[b]:bs[b + 1]] = pm[d, bs[b]:bs[b + 1]]
    AF = np.kron(np.eye(3), af)
    Z2 = np.zeros((nb, N))
    AM = np.block([[Z2, -x_m[2], x_m[1]], [x_m[2], Z2, -x_m[0]], [-x_m[1], x_m[0], Z2]])
    B = np.vstack([AF, AM])
    BT = np.hstack([AU, AOm])
    return B, BT, B @ B.T, BT.T @ BT


def interleaved_to_blocked(N):
    """Permutation matrix P with P @ v_interleaved = v_blocked for 3N vectors."""
    idx = np.arange(3 * N).reshape(N, 3).T.ravel()
    P = np.zeros((3 * N, 3 * N))
    P[np.arange(3 * N), idx] = 1.0
    return P


def dense_velocity_operator(asm, eps, mu, nearest):
    """S*kron(NN,I3) (or S) in the blocked layout: the exact operator that
    FMM.computeVel approximates with 'GMRES',1,'format',2."""
    pts = asm["points"]
    N = len(pts)
    if nearest:
        S = kernel(asm["fine"], pts, eps, mu) @ np.kron(asm["NN"].toarray(), np.eye(3))
    else:
        S = kernel(pts, pts, eps, mu)
    P = interleaved_to_blocked(N)
    return P @ S @ P.T


def mobility_rhs(asm, fluid=None):
    """input of mobilityProblem.m:37-46.  The background velocity is
    subtracted on the swimmer rows only (:40-41)."""
    vel = asm["vel"].copy()
    if fluid is not None:
        Nsw = asm["bstart"][-1]
        vel[:Nsw] -= fluid(asm["points"][:Nsw])
    F, M = asm["Fsw"], asm["Msw"]
    return np.concatenate([vel.T.ravel(), F[:, 0], F[:, 1], F[:, 2], M[:, 0], M[:, 1], M[:, 2]])


def dense_mobility_matrix(asm, eps, mu, nearest):
    A = dense_velocity_operator(asm, eps, mu, nearest)
    B, BT, _, _ = gen_matrix_components(asm, nearest)
    nb6 = 6 * asm["nb"]
    return np.block([[A, BT], [B, np.zeros((nb6, nb6))]])


def rigid_output(asm, x, bodies):
    """out = [U; Om x b1; Om x b2] per body (mobilityProblem.m:60-72)."""
    nb = asm["nb"]
    U = x[-6 * nb:-3 * nb].reshape(3, nb).T
    Om = x[-3 * nb:].reshape(3, nb).T
    out = []
    for i, b in enumerate(bodies):
        out.extend([U[i], np.cross(Om[i], b.b1), np.cross(Om[i], b.b2)])
    return np.concatenate(out) if out else np.zeros(0)


def mobility_precon(f, asm, fmm, nearest=True):
    r"""The block preconditioner of Mobility/MobilityPrecon.m:17-39 applied to
    f = [force (3N, blocked x|y|z); U (3 nb); Omega (3 nb)].

    ``fmm`` is an oracle KIFMM (``gmres=1, fmt=2``, the blocked vector layout
    MobilityPrecon.m:26 selects) on the swimmers' tree (all force points,
    NEAREST with the block NN):
      b(force) = reducedSolve(force)                                  (:29-30)
      out      = -A2 \ (BT' * computeVelSparse(B' * (A1 \ UOm)))      (:32-34)
      b(force) = b(force) - reducedSolve(BT * out)                     (:38-39)
    with [B, BT, A1, A2] of genMatrixComponets.m (dense here)."""
    nb = asm["nb"]
    f = np.asarray(f, dtype=np.float64).ravel()
    force, UOm = f[:-6 * nb], f[-6 * nb:]
    B, BT, A1, A2 = gen_matrix_components(asm, nearest)
    b = np.zeros_like(f)
    b[:-6 * nb] = fmm.reduced_solve(force)
    out = -np.linalg.solve(A2, BT.T @ fmm.compute_vel_sparse(B.T @ np.linalg.solve(A1, UOm)))
    b[-6 * nb:] = out
    b[:-6 * nb] -= fmm.reduced_solve(BT @ out)
    return b
