"""Rigid-body resistance problems (Resistance/Rigid_Resistance.m:18-43,
Resistance/Gen_Resistance.m:12-26, Geometries/velocityModes.m:13-25).

For a prescribed rigid motion (velocity U, angular velocity Omega) the point
velocities u = U + Omega x X at the force points are imposed, the first-kind
system S kron(NN, I3) f = u is solved by GMRES on the device FMM
(nnk_fmm_solve; the reference's Rigid_Resistance.m:24 calls `this.computeVel`,
which is not defined there: the KIFMM passed in is meant), and the total force
and moment are returned:
  F = sum over fine points of kron(NN, I3) f          (Rigid_Resistance.m:27-29, 37)
  M = sum over force points of x_n x f_n,  x_n = sum_q NN(q, n) X_q
      (NN-weighted sums of the fine positions, :31-33, 40-43);
in plain mode the sums run over the force points themselves.  Gen_Resistance
stacks the six unit modes into the 6 x 6 grand resistance matrix
[[F_U, F_Omega], [M_U, M_Omega]].
"""
import numpy as np

__all__ = ["velocityModes", "Rigid_Resistance", "Gen_Resistance", "force_moment"]


def velocityModes(points, vel, mom):
    """U + Omega x X per point (N x 3); Geometries/velocityModes.m:13-25."""
    p = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    U = np.asarray(vel, dtype=np.float64).ravel()
    W = np.asarray(mom, dtype=np.float64).ravel()
    return U[None, :] + np.cross(W[None, :], p)


def _layout_vec(fmm, rows):
    """(N, 3) rows in the FMM's GMRES vector format (1: interleaved, 2: blocked)."""
    return rows.T.ravel() if fmm.arguments.get("format", 1) == 2 else rows.ravel()


def _rows(fmm, v):
    v = np.asarray(v, dtype=np.float64).ravel()
    return v.reshape(3, -1).T if fmm.arguments.get("format", 1) == 2 else v.reshape(-1, 3)


def Rigid_Resistance(fmm, vel, mom, tol=1e-6, maxIter=None):
    """Total force F (3,) and moment M (3,) on the body of `fmm` moving
    rigidly with velocity `vel` and angular velocity `mom`, with the GMRES
    outputs: returns (F, M, flag, relres, iters)."""
    tree = fmm.tree
    X = tree.points[tree.targets]
    u = velocityModes(X, vel, mom)
    f, flag, relres, it = fmm.gmres(_layout_vec(fmm, u), tol=tol, maxit=maxIter)
    F, M = force_moment(_rows(fmm, f), X, tree.NN, tree.finePoints)
    return F, M, flag, relres, it


def force_moment(f, X, NN=None, fine=None):
    """Total force and moment of the force densities f (N x 3) at the force
    points X: with NEAREST (NN, fine given) F = sum_q (NN f)_q and
    M = sum_n x_n x f_n, x_n = sum_q NN(q, n) fine_q; else sums over X."""
    f = np.asarray(f, dtype=np.float64).reshape(-1, 3)
    if NN is not None:
        F = np.asarray(NN @ f).sum(axis=0)
        x = np.asarray(NN.T @ np.asarray(fine, dtype=np.float64))
    else:
        F = f.sum(axis=0)
        x = np.asarray(X, dtype=np.float64)
    return F, np.cross(x, f).sum(axis=0)


def Gen_Resistance(fmm, tol=1e-6, maxIter=None):
    """The 6 x 6 grand resistance matrix R = [[F_U, F_Om], [M_U, M_Om]]
    (column j: unit velocity e_j for j < 3, unit angular velocity e_{j-3});
    Gen_Resistance.m:12-26."""
    R = np.zeros((6, 6))
    for j in range(6):
        vel, mom = np.zeros(3), np.zeros(3)
        (vel if j < 3 else mom)[j % 3] = 1.0
        F, M, flag, relres, it = Rigid_Resistance(fmm, vel, mom, tol=tol, maxIter=maxIter)
        if flag != 0:
            raise RuntimeError(f"resistance GMRES stopped at relres {relres:.3e} after {it} iterations")
        R[:3, j] = F
        R[3:, j] = M
    return R
