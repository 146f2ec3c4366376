"""Differentiable rigid-body mobility through torch.autograd.

`rigid_velocity(X, Y, eps, F, M)` returns [U; Omega] of one free body with
force points X (N x 3) and quadrature points Y (Q x 3) under a force F and a
torque M (mobilityProblem.m:37-72 with zero slip, body at rest orientation,
centre x0 = 0), and is differentiable with respect to X, Y and eps.

Forward: NEAREST tree, KIFMM and device GMRES (nnk_mob_solve), the
reference's path.  Backward, for a loss L(z) of the solution z = [f; U; Om]:
  * the adjoint system A^T lam = dL/dz is solved by GMRES on the device with
    the exact transpose of the FMM (nnk_mob_solve_adjoint);
  * dL/dX and dL/dY = -lam^T (dA/dpositions) z come from the kernel's
    derivative evaluated through the FMM's leaf stages and the rigid-body
    blocks (nnk_mob_grad_positions); NN is held fixed (piecewise constant in
    the positions);
  * dL/deps = -lam^T (dA/deps) z by the analytic eps-derivative of the FMM
    (nnk_mob_grad_eps): the kernel's eps-derivative in every pair sum and in
    the M2L, and d(K^-1)/deps of the check-to-equivalent solves, contracted
    with the forward and transpose passes' quantities, on an FP64 FMM with
    the exact inverses (the mobility object's own in FP64 mode).  With
    Tikhonov operators (reg > 0) it is the central difference of two FP64
    matvecs at eps (1 +- 1e-3) instead.
In mixed precision the solves use FP32 pairs with FP64 refinement.
"""
import numpy as np
import torch

from .kifmm import KIFMM
from .mobility import Swimmers, mobilityRHS
from .octree import nearestMatrix


class _RigidVelocity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, X, Y, eps, F, M, opts):
        Xn = X.detach().cpu().numpy().astype(np.float64)
        Yn = Y.detach().cpu().numpy().astype(np.float64)
        e = float(eps.detach().cpu())
        mu = opts["mu"]
        NN = nearestMatrix(Xn, Yn)
        sw = Swimmers()
        sw.addSwimmer(Xn, Yn, NN, [0.0, 0.0, 0.0], [1, 0, 0, 0, 1, 0], np.zeros_like(Xn),
                      np.asarray(F, float), np.asarray(M, float))
        sw.genTree(nodeCapacity=opts["cap"], nearest=1)
        kw = dict(GMRES=1, format=2, precision=opts["precision"])
        if opts["reg"] > 0:
            kw["reg"] = opts["reg"]
        sw.genKIFMM([e, mu], **kw)
        mob = sw.mobility()
        z, flag, relres, it = mob.solve(mobilityRHS(sw), tol=opts["tol"], maxIter=opts["maxIter"])
        if flag != 0:
            raise RuntimeError(f"mobility GMRES stopped at relres {relres:.3e} after {it} iterations")
        ctx.state = (sw, mob, z, e, opts)
        ctx.info = dict(iters=it, relres=relres)
        return torch.as_tensor(z[-6:].copy(), dtype=X.dtype, device=X.device)

    @staticmethod
    def backward(ctx, gout):
        sw, mob, z, e, opts = ctx.state
        g = np.zeros(mob.n)
        g[-6:] = gout.detach().cpu().numpy().astype(np.float64)
        lam, flag, relres, it = mob.solve_adjoint(g, tol=opts["tol"], maxIter=opts["maxIter"])
        if flag != 0:
            raise RuntimeError(f"adjoint GMRES stopped at relres {relres:.3e} after {it} iterations")
        gX, gY = mob.grad_positions(z, lam)
        if opts["reg"] > 0:
            # Tikhonov operators: a central difference of two FP64 matvecs
            d = 1e-3 * e
            f64 = KIFMM(sw.Tree, [e, opts["mu"]], GMRES=1, format=2, precision="fp64", reg=opts["reg"])
            f64.setEps(e + d)
            Ap = mob.apply_with(f64, z)
            f64.setEps(e - d)
            Am = mob.apply_with(f64, z)
            geps = -float(lam @ (Ap - Am)) / (2 * d)
        else:
            exact = None if opts["precision"] == "fp64" else \
                KIFMM(sw.Tree, [e, opts["mu"]], GMRES=1, format=2, precision="fp64")
            geps = mob.grad_eps(z, lam, exact)
        ctx.grad_info = dict(iters=it, relres=relres)
        X_dtype, dev = gout.dtype, gout.device
        return (torch.as_tensor(gX, dtype=X_dtype, device=dev), torch.as_tensor(gY, dtype=X_dtype, device=dev),
                torch.tensor(geps, dtype=X_dtype, device=dev), None, None, None)


def rigid_velocity(X, Y, eps, F, M, mu=1.0, cap=60, precision="fp64", tol=1e-10, maxIter=500, reg=0.0):
    """[U; Omega] (6,) of the body, differentiable in X, Y and eps (torch
    tensors).  reg > 0 uses Tikhonov check-to-equivalent operators in FP64
    mode as well (smaller rounding, for finite-difference checks)."""
    if not torch.is_tensor(eps):
        eps = torch.tensor(float(eps), dtype=X.dtype)
    opts = dict(mu=float(mu), cap=int(cap), precision=precision, tol=float(tol), maxIter=int(maxIter),
                reg=float(reg))
    return _RigidVelocity.apply(X, Y, eps, np.asarray(F, float), np.asarray(M, float), opts)
