"""Swimmers container and the GMRES mobility solve, host mirror of
Classes/Swimmers.m and Mobility/mobilityProblem.m over the CUDA library.

    sw = Swimmers()
    sw.addSwimmer(points, fine, NN, x0, b1b2, vel, F, M)      # NEAREST form
    out = mobilityProblem(sw, fluidFunc, t, conditions, [eps, mu],
                          {'nodeCapacity': 60, 'nearest': 1}, tol=1e-6, maxIter=100)

The mobility matvec (Mobility/MobilityMatrixMulti.m), the block
preconditioner (Mobility/MobilityPrecon.m) and GMRES run on the device
through nnk_mob_*; this module only assembles the geometry and right-hand
side the way Swimmers.m does.
"""
import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _lib as L
from .kifmm import KIFMM
from .octree import OcTree


def _basis(b1, b2):
    b1 = np.asarray(b1, float).ravel()
    b2 = np.asarray(b2, float).ravel()
    return np.stack([b1, b2, np.cross(b1, b2)], axis=1)


class Swimmers:
    """Classes/Swimmers.m: per-body geometry in the body frame, centre x0,
    basis (b1,b2), slip velocity, total force and moment, plus a boundary."""

    def __init__(self):
        self.x0, self.b, self.Geometries, self.Vel = [], [], [], []
        self.GeometriesFine, self.NN, self.F, self.Moment = [], [], [], []
        self.Boundary = np.zeros((0, 3))
        self.BoundaryVel = np.zeros((0, 3))
        self.BoundaryFine = np.zeros((0, 3))
        self.BoundaryNN = None
        self.Tree = None
        self.FMM = None
        self.mob = None

    def addSwimmer(self, *args):
        """(points, centre, basis, vel, F, M) or
        (points, fine, NN, centre, basis, vel, F, M) (Swimmers.m:83-125)."""
        if len(args) == 6:
            pts, x0, b, vel, F, M = args
            fine, NN = None, None
        elif len(args) == 8:
            pts, fine, NN, x0, b, vel, F, M = args
        else:
            raise ValueError("Invalid number of inputs")
        b = np.asarray(b, float).ravel()
        self.Geometries.append(np.asarray(pts, float))
        self.GeometriesFine.append(None if fine is None else np.asarray(fine, float))
        self.NN.append(None if NN is None else sp.csr_matrix(NN))
        self.x0.append(np.asarray(x0, float).ravel())
        self.b.append((b[0:3].copy(), b[3:6].copy()))
        self.Vel.append(np.asarray(vel, float))
        self.F.append(np.asarray(F, float).ravel())
        self.Moment.append(np.asarray(M, float).ravel())

    def updateBnd(self, *args):
        """(points, vel) or (points, fine, NN, vel) (Swimmers.m:127-148)."""
        if len(args) == 2:
            self.Boundary, self.BoundaryVel = np.asarray(args[0], float), np.asarray(args[1], float)
            self.BoundaryFine, self.BoundaryNN = np.zeros((0, 3)), None
        elif len(args) == 4:
            self.Boundary = np.asarray(args[0], float)
            self.BoundaryFine = np.asarray(args[1], float)
            self.BoundaryNN = sp.csr_matrix(args[2])
            self.BoundaryVel = np.asarray(args[3], float)
        else:
            raise ValueError("Invalid number of inputs")

    def swimmerNo(self):
        return len(self.Geometries)

    def getSwimmerSizes(self):
        return ([len(g) for g in self.Geometries],
                [0 if f is None else len(f) for f in self.GeometriesFine])

    def _rot(self):
        return [_basis(b1, b2) for b1, b2 in self.b]

    def getSwimmers(self):
        """(points, finePoints, NN, pointsrot, finerot) (Swimmers.m:150-200)."""
        Bs = self._rot()
        rel = [(B @ g.T).T for B, g in zip(Bs, self.Geometries)]
        pts = [r + x0 for r, x0 in zip(rel, self.x0)]
        frel = [(B @ f.T).T for B, f in zip(Bs, self.GeometriesFine) if f is not None]
        fine = [(B @ f.T).T + x0 for B, f, x0 in zip(Bs, self.GeometriesFine, self.x0) if f is not None]
        nns = [n for n in self.NN if n is not None]
        cat = lambda a: np.concatenate(a) if a else np.zeros((0, 3))
        return (cat(pts), cat(fine), sp.block_diag(nns, format="csr") if nns else None, cat(rel), cat(frel))

    def getSwimmerBnd(self):
        """Swimmers first, then the boundary (Swimmers.m:254-310)."""
        pts, fine, NN, _, _ = self.getSwimmers()
        P = np.concatenate([pts, self.Boundary]) if len(self.Boundary) else pts
        Fp = np.concatenate([fine, self.BoundaryFine]) if len(self.BoundaryFine) else fine
        blocks = [m for m in [NN, self.BoundaryNN] if m is not None]
        return P, Fp, (sp.block_diag(blocks, format="csr") if blocks else None)

    def getVelocities(self):
        """Rotated slip velocities then the boundary's (Swimmers.m:312-340)."""
        v = [(B @ u.T).T for B, u in zip(self._rot(), self.Vel)]
        v = np.concatenate(v) if v else np.zeros((0, 3))
        return np.concatenate([v, self.BoundaryVel]) if len(self.BoundaryVel) else v

    def getForceMoment(self):
        return np.concatenate(self.F), np.concatenate(self.Moment)

    def updateSwimmmer(self, index, x0, b):
        """index is 1-based as in Swimmers.m:361-370."""
        b = np.asarray(b, float).ravel()
        self.x0[index - 1] = np.asarray(x0, float).ravel()
        self.b[index - 1] = (b[0:3].copy(), b[3:6].copy())

    def updateSwimmmerRHS(self, index, G, offset):
        """Gravity forcing F = G, M = -4/3 pi offset (b3 x G) (Swimmers.m:372-385)."""
        b1, b2 = self.b[index - 1]
        b3 = np.cross(b1, b2)
        G = np.asarray(G, float).ravel()
        self.F[index - 1] = G.copy()
        self.Moment[index - 1] = -4.0 / 3.0 * np.pi * offset * np.cross(b3, G)

    def genTree(self, **treePar):
        """OcTree(points, points, 'finePoints', fine, 'NN', NN, ...) (Swimmers.m:387-398)."""
        P, Fp, NN = self.getSwimmerBnd()
        self.Tree = OcTree(P, P, finePoints=Fp if len(Fp) else None, NN=NN, **treePar)
        return self

    def genKIFMM(self, kernelPar, refine=None, **kw):
        """KIFMM on the current tree (Swimmers.m:400-410).  With
        precision='mixed', refine=True (the default for mixed) also builds an
        FP64 KIFMM used for the outer residuals of iterative refinement."""
        if kw.get("precision", "fp64") == "mixed":
            # Mobility systems are ill-conditioned (kappa ~ 1e4); the TF32
            # rounding of tensor-core M2L (~4e-5) then stalls GMRES near 1e-5
            # and slows refinement, so solves default to an M2L with FP32
            # accuracy: the Fourier-space product (4x fewer flops than the
            # FP32 pair kernel).
            kw.setdefault("m2l", "fft")
        self.FMM = KIFMM(self.Tree, kernelPar, **kw)
        self.FMM64 = None
        if kw.get("precision", "fp64") == "mixed" and refine is not False:
            # the outer residual uses FP64 arithmetic on the same regularized
            # check-to-equivalent operators, so the two operators differ by
            # rounding only and the refinement contracts quickly
            kw64 = dict(kw)
            kw64["precision"] = "fp64"
            kw64.pop("m2l", None)
            kw64["reg"] = kw.get("reg", 0.0) or 1e-5
            self.FMM64 = KIFMM(self.Tree, kernelPar, **kw64)
        self.mob = None
        return self

    def mobility(self):
        """Device mobility operator on the current tree and FMM."""
        if self.mob is None:
            self.mob = Mobility(self)
        return self.mob


class Mobility:
    """nnk_mob_* wrapper: matvec (MobilityMatrixMulti.m), preconditioner
    (MobilityPrecon.m) and GMRES (mobilityProblem.m:48-58)."""

    def __init__(self, sw):
        self.sw = sw
        fmm = sw.FMM
        sizes, fsizes = sw.getSwimmerSizes()
        bstart = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        fstart = np.concatenate([[0], np.cumsum(fsizes)]).astype(np.int64)
        _, _, _, rel, frel = sw.getSwimmers()
        rel = np.ascontiguousarray(rel) if len(rel) else np.zeros((1, 3))
        frel = np.ascontiguousarray(frel) if len(frel) else np.zeros((1, 3))
        h = C.c_void_p()
        L.check(L.lib.nnk_mob_create(fmm.h, len(sizes), L.ptr(bstart), L.ptr(fstart), L.ptr(rel), L.ptr(frel),
                                     C.byref(h)), fmm.ctx.h, "mobility")
        self.h = h
        self.fmm = fmm  # the native operator refers to it
        self.ctx = fmm.ctx
        self.n = 3 * fmm.tree.info.num_targets + 6 * len(sizes)
        if getattr(sw, "FMM64", None) is not None:
            self.set_refinement(sw.FMM64)

    def set_refinement(self, fmm64, max_outer=12, inner_tol=1e-3):
        """Mixed-precision iterative refinement against an FP64 KIFMM on the same tree."""
        self.fmm64 = fmm64
        L.check(L.lib.nnk_mob_set_refinement(self.h, fmm64.h if fmm64 is not None else None, int(max_outer),
                                             float(inner_tol)), self.ctx.h, "refinement")

    _destroy = L.lib.nnk_mob_destroy  # held by the class: module globals may be gone at exit

    def __del__(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def _vec(self, x):
        x = np.ascontiguousarray(np.asarray(x, float).ravel())
        if x.size != self.n:
            raise ValueError(f"expected a vector of {self.n}")
        return x

    def apply(self, x):
        x = self._vec(x)
        y = np.empty(self.n)
        L.check(L.lib.nnk_mob_apply(self.h, L.ptr(x), L.ptr(y), 0), self.ctx.h, "mobilityMatrixMulti")
        return y

    def apply_adjoint(self, x):
        """A^T x (the transpose of mobilityMatrixMulti)."""
        x = self._vec(x)
        y = np.empty(self.n)
        L.check(L.lib.nnk_mob_apply_adjoint(self.h, L.ptr(x), L.ptr(y), 0), self.ctx.h, "adjoint")
        return y

    def apply_with(self, fmm, x):
        """The matvec with another KIFMM on the same tree."""
        x = self._vec(x)
        y = np.empty(self.n)
        L.check(L.lib.nnk_mob_apply_fmm(self.h, fmm.h, L.ptr(x), L.ptr(y), 0), self.ctx.h, "apply_with")
        return y

    def solve_adjoint(self, rhs, tol=1e-6, maxIter=None, restart=0):
        rhs = self._vec(rhs)
        x = np.empty(self.n)
        sp_ = L.SolveParams(float(tol), int(maxIter if maxIter else min(self.n, 10)), int(restart))
        info = L.SolveInfo()
        rc = L.lib.nnk_mob_solve_adjoint(self.h, L.ptr(rhs), L.ptr(x), C.byref(sp_), C.byref(info), 0)
        if rc not in (L.NNK_OK, L.NNK_E_NOCONV):
            L.check(rc, self.ctx.h, "adjoint gmres")
        return x, info.flag, info.relres, info.iters

    def grad_positions(self, z, lam):
        """-lam^T (dA/dpositions) z: (N x 3 force points, Q x 3 fine points)."""
        z, lam = self._vec(z), self._vec(lam)
        info = self.sw.Tree.info
        gx = np.empty((info.num_targets, 3))
        gy = np.empty((max(info.num_fine, 0), 3))
        L.check(L.lib.nnk_mob_grad_positions(self.h, L.ptr(z), L.ptr(lam), L.ptr(gx),
                                             L.ptr(gy) if info.num_fine else None, 0), self.ctx.h, "gradient")
        return gx, gy

    def grad_eps(self, z, lam, fmm64=None):
        """-lam^T (dA/deps) z through the analytic eps-derivative of the FMM
        (nnk_mob_grad_eps); fmm64: an FP64 KIFMM with the exact
        check-to-equivalent inverses on the same tree, when this object's own
        FMM is not one."""
        z, lam = self._vec(z), self._vec(lam)
        out = C.c_double()
        L.check(L.lib.nnk_mob_grad_eps(self.h, fmm64.h if fmm64 is not None else None, L.ptr(z), L.ptr(lam),
                                       C.byref(out), 0), self.ctx.h, "grad_eps")
        return out.value

    def use_graphs(self, enable=True):
        """Replay the matvec from a CUDA graph (default) or launch kernel by kernel."""
        L.check(L.lib.nnk_mob_use_graphs(self.h, int(bool(enable))), self.ctx.h, "use_graphs")

    def precon(self, x):
        x = self._vec(x)
        y = np.empty(self.n)
        L.check(L.lib.nnk_mob_precon(self.h, L.ptr(x), L.ptr(y), 0), self.ctx.h, "mobilityPrecon")
        return y

    def solve(self, rhs, tol=1e-6, maxIter=None, precondition=False, restart=0, x0=None):
        """gmres(afunc, rhs, restart, tol, maxIter[, ..., x0]) on the device.
        With an initial guess x0 (MATLAB's 8th gmres argument, used by the
        reference's Hegedus-trick experiments, Tests/HegadusTrickTest.m and
        Data Generation/preconditioningInitalGuess.m) the correction
        d = A^-1 (rhs - A x0) is solved from zero to the tolerance that makes
        ||rhs - A (x0 + d)|| / ||rhs|| <= tol, and x0 + d is returned."""
        if x0 is not None:
            rhs = self._vec(rhs)
            x0 = self._vec(x0)
            r0 = rhs - self.apply(x0)
            nb, nr = float(np.linalg.norm(rhs)), float(np.linalg.norm(r0))
            if nb == 0.0 or nr <= tol * nb:
                return x0.copy(), 0, (nr / nb if nb else 0.0), 0
            d, flag, relres, it = self.solve(r0, tol=tol * nb / nr, maxIter=maxIter, precondition=precondition,
                                             restart=restart)
            return x0 + d, flag, relres * nr / nb, it
        rhs = self._vec(rhs)
        x = np.empty(self.n)
        sp_ = L.SolveParams(float(tol), int(maxIter if maxIter else min(self.n, 10)), int(restart))
        info = L.SolveInfo()
        rc = L.lib.nnk_mob_solve(self.h, L.ptr(rhs), L.ptr(x), C.byref(sp_), int(bool(precondition)),
                                 C.byref(info), 0)
        if rc not in (L.NNK_OK, L.NNK_E_NOCONV):
            L.check(rc, self.ctx.h, "gmres")
        return x, info.flag, info.relres, info.iters


def hegedus(apply, b, xp):
    """The Hegedus trick (Tests/HegadusTrickTest.m, preconditioningInitalGuess.m:
    scale = (b' A xp) / ||A xp||^2): the multiple of a previous solution xp (of
    a nearby system, e.g. another eps) that minimises ||b - A x0||, as the
    initial guess x0 = scale * xp."""
    b = np.asarray(b, dtype=np.float64).ravel()
    xp = np.asarray(xp, dtype=np.float64).ravel()
    Axp = np.asarray(apply(xp), dtype=np.float64).ravel()
    den = float(Axp @ Axp)
    return (float(b @ Axp) / den if den > 0 else 0.0) * xp


def mobilityRHS(sw, fluidFunc=None, t=0.0):
    """input of mobilityProblem.m:37-46 (background flow subtracted on the
    swimmer rows only, as :40-41 do)."""
    vel = sw.getVelocities().copy()
    if fluidFunc is not None:
        pts = sw.getSwimmers()[0]
        vel[:len(pts)] -= fluidFunc(t, pts)
    force, moment = sw.getForceMoment()
    return np.concatenate([vel.T.ravel(), force[0::3], force[1::3], force[2::3],
                           moment[0::3], moment[1::3], moment[2::3]])


def mobilityProblem(swimmers, fluidFunc, t, conditions, kernelPar, TreePar, threads=0, GPU=1,
                    blockSize=0.1, tol=1e-6, maxIter=None, PreconSettings=None, precision="fp64",
                    return_info=False, refine=None):
    """Mobility/mobilityProblem.m:1-72.  conditions = (9*nb) [x0; b1; b2] per
    body; returns (9*nb) [U; Om x b1; Om x b2] per body."""
    conditions = np.asarray(conditions, float).ravel()
    nb = conditions.size // 9
    for i in range(nb):
        d = conditions[9 * i:9 * i + 9]
        swimmers.updateSwimmmer(i + 1, d[0:3], d[3:9])
    swimmers.genTree(**dict(TreePar))
    swimmers.genKIFMM(kernelPar, refine=refine, parThreads=threads, GPU=GPU, GMRES=1, format=2,
                      blockSize=blockSize, precision=precision)
    mob = swimmers.mobility()
    rhs = mobilityRHS(swimmers, fluidFunc, t)
    x, flag, relres, it = mob.solve(rhs, tol=tol, maxIter=maxIter, precondition=bool(PreconSettings is not None
                                                                                     and len(PreconSettings)))
    U = x[-6 * nb:-3 * nb].reshape(3, nb).T
    Om = x[-3 * nb:].reshape(3, nb).T
    out = np.zeros(9 * nb)
    for i in range(nb):
        b1, b2 = swimmers.b[i]
        out[9 * i:9 * i + 3] = U[i]
        out[9 * i + 3:9 * i + 6] = np.cross(Om[i], b1)
        out[9 * i + 6:9 * i + 9] = np.cross(Om[i], b2)
    if return_info:
        return out, dict(flag=flag, relres=relres, iters=it, x=x)
    return out


def mobilityProblemGravity(swimmers, fluidFunc, t, conditions, kernelPar, TreePar, threads=0, GPU=1,
                           blockSize=0.1, tol=1e-6, maxIter=None, PreconSettings=None, gravPar=(0, 0, -1, 0),
                           precision="fp64", return_info=False, refine=None):
    """Mobility/mobilityProblemGravity.m:1-74: mobilityProblem with every
    swimmer forced by gravity, F = G and M = -4/3 pi offset (b3 x G) for
    gravPar = [G (3); offset] (Swimmers.m:372-385), set after its centre and
    basis are updated from `conditions`."""
    conditions = np.asarray(conditions, float).ravel()
    g = np.asarray(gravPar, float).ravel()
    for i in range(conditions.size // 9):
        d = conditions[9 * i:9 * i + 9]
        swimmers.updateSwimmmer(i + 1, d[0:3], d[3:9])
        swimmers.updateSwimmmerRHS(i + 1, g[0:3], g[3])
    return mobilityProblem(swimmers, fluidFunc, t, conditions, kernelPar, TreePar, threads, GPU, blockSize, tol,
                           maxIter, PreconSettings, precision, return_info, refine)


def richardson(values, eps):
    """Extrapolation to eps -> 0 of results at two regularisation widths,
    assuming an O(eps) error (the regularized Stokeslet's leading term):
    (e1 v2 - e2 v1) / (e1 - e2)."""
    (v1, v2), (e1, e2) = values, eps
    v1, v2 = np.asarray(v1, float), np.asarray(v2, float)
    return (e1 * v2 - e2 * v1) / (e1 - e2)
