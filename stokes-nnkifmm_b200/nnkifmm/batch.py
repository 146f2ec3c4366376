"""Many independent rigid-body mobility problems solved together.

Each body gets its own device context (its own CUDA stream), NEAREST tree,
KIFMM (mixed precision with FP64 refinement, or FP64) and mobility operator;
host threads drive the bodies concurrently so that the kernels of different
bodies overlap on the GPU, and each body's 6 rigid-mode right-hand sides
(unit forces and unit torques, the columns of Resistance/Gen_Resistance.m's
modes in mobility form) are solved one after another on its stream.
"""
import concurrent.futures as cf

import numpy as np

from . import _lib as L
from .mobility import Swimmers, mobilityRHS
from .octree import nearestMatrix

RIGID_MODES = [("F", 0), ("F", 1), ("F", 2), ("M", 0), ("M", 1), ("M", 2)]


class Body:
    def __init__(self, coarse, fine, kernelPar, cap, precision, device, preconditioned, refine=None, m2l="pairs"):
        self.ctx = L.Context(device)
        self.coarse, self.fine = coarse, fine
        NN = nearestMatrix(coarse, fine)
        self.sw = Swimmers()
        self.sw.addSwimmer(coarse, fine, NN, [0.0, 0.0, 0.0], [1, 0, 0, 0, 1, 0], np.zeros_like(coarse),
                           [0.0, 0.0, 0.0], [0.0, 0.0, 0.0])
        self.sw.genTree(nodeCapacity=cap, nearest=1, ctx=self.ctx)
        kw = dict(GMRES=1, format=2, precision=precision)
        if precision == "mixed":
            kw["m2l"] = m2l
        self.sw.genKIFMM(kernelPar, refine=refine, **kw)
        self.mob = self.sw.mobility()
        self.preconditioned = preconditioned

    def rhs(self, mode):
        kind, k = mode
        F = np.zeros(3)
        M = np.zeros(3)
        (F if kind == "F" else M)[k] = 1.0
        self.sw.F[0], self.sw.Moment[0] = F, M
        return mobilityRHS(self.sw)

    def solve_modes(self, tol, maxIter, modes=RIGID_MODES):
        """6 x 6 mobility matrix of the body: column j = [U; Omega] for mode j."""
        out = np.zeros((6, len(modes)))
        iters = []
        for j, m in enumerate(modes):
            x, flag, relres, it = self.mob.solve(self.rhs(m), tol=tol, maxIter=maxIter,
                                                 precondition=self.preconditioned)
            out[:, j] = x[-6:]
            iters.append((flag, relres, it))
        return out, iters


class BatchMobility:
    def __init__(self, bodies, kernelPar, cap=200, precision="mixed", device=0, workers=8,
                 preconditioned=False, refine=None, m2l="pairs"):
        self.workers = workers
        with cf.ThreadPoolExecutor(max_workers=workers) as ex:
            self.bodies = list(ex.map(lambda b: Body(b[0], b[1], kernelPar, cap, precision, device,
                                                     preconditioned, refine, m2l), bodies))

    def solve_all(self, tol=1e-6, maxIter=200, modes=RIGID_MODES):
        with cf.ThreadPoolExecutor(max_workers=self.workers) as ex:
            res = list(ex.map(lambda b: b.solve_modes(tol, maxIter, modes), self.bodies))
        return [r[0] for r in res], [r[1] for r in res]
