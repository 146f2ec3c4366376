"""Many independent rigid-body mobility problems.

`Body` is one body solved the reference's way: its own NEAREST tree, KIFMM
and mobility operator, one gmres call per right-hand side
(mobilityProblem.m:53).  `BatchMobility` solves all bodies and all their
right-hand sides together through nnk_batch_*: the bodies' trees form one
forest, one FMM pass evaluates every body and every right-hand side (the pair
kernels share the geometry of a pair across a body's right-hand sides), and
GMRES runs per system with all systems advancing in lockstep.

The right-hand sides of `solve_modes` are the 6 rigid modes in mobility form:
unit force or unit torque, no slip (the columns of Gen_Resistance.m's modes),
so the result per body is its 6 x 6 mobility matrix.
"""
import ctypes as C

import numpy as np

from . import _lib as L
from .mobility import Swimmers, mobilityRHS
from .octree import OcTree, nearestMatrix

RIGID_MODES = [("F", 0), ("F", 1), ("F", 2), ("M", 0), ("M", 1), ("M", 2)]


def mode_rhs(n_points, mode):
    """[f (3N) = 0 | F | M] with the unit force or torque of `mode`."""
    kind, k = mode
    v = np.zeros(3 * n_points + 6)
    v[3 * n_points + (0 if kind == "F" else 3) + k] = 1.0
    return v


class Body:
    """One body through the per-body path (Swimmers + KIFMM + nnk_mob)."""

    def __init__(self, coarse, fine, kernelPar, cap, precision, device=0, preconditioned=False, refine=None,
                 m2l="fft", ctx=None):
        self.ctx = ctx if ctx is not None else L.Context(device)
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
    """All bodies x nrhs right-hand sides in one batch (nnk_batch_*).

    bodies: list of (force points N_b x 3, fine points Q_b x 3), each a free
    body at rest orientation (rel points = the points themselves).
    precision 'mixed' uses FP32 pair kernels and an FP32 M2L (m2l='fft':
    Fourier-space product, 'pairs': pair kernel) with FP64 iterative
    refinement unless refine=False."""

    def __init__(self, bodies, kernelPar, cap=200, precision="mixed", nrhs=6, refine=None, device=0, ctx=None,
                 max_outer=12, inner_tol=1e-4, m2l="fft"):
        self.ctx = ctx if ctx is not None else L.Context(device)
        self.nrhs = int(nrhs)
        self.sizes = []
        trees, rel, frel = [], [], []
        for coarse, fine in bodies:
            coarse = np.ascontiguousarray(coarse, dtype=np.float64)
            fine = np.ascontiguousarray(fine, dtype=np.float64)
            NN = nearestMatrix(coarse, fine)
            trees.append(OcTree(coarse, coarse, nodeCapacity=cap, finePoints=fine, nearest=1, NN=NN, ctx=self.ctx))
            rel.append(coarse)
            frel.append(fine)
            self.sizes.append(len(coarse))
        nb = len(trees)
        th = (C.c_void_p * nb)(*[t.h for t in trees])
        rp = (C.c_void_p * nb)(*[a.ctypes.data for a in rel])
        fp = (C.c_void_p * nb)(*[a.ctypes.data for a in frel])
        prec = L.PREC_MIXED if precision == "mixed" else L.PREC_FP64
        mode = {"fft": 4, "pairs": 3}[m2l] if prec == L.PREC_MIXED else 0
        params = L.FmmParams(float(kernelPar[0]), float(kernelPar[1]), 6, 1, prec, mode, 0.0)
        h = C.c_void_p()
        L.check(L.lib.nnk_batch_create(self.ctx.h, nb, th, rp, fp, C.byref(params), self.nrhs, C.byref(h)),
                self.ctx.h, "nnk_batch_create")
        self.h = h
        n = C.c_int64()
        self.offsets = np.zeros(nb * self.nrhs + 1, np.int64)
        L.check(L.lib.nnk_batch_layout(self.h, C.byref(n), L.ptr(self.offsets)))
        self.n = n.value
        if prec == L.PREC_MIXED and refine is not False:
            L.check(L.lib.nnk_batch_set_refinement(self.h, 1, int(max_outer), float(inner_tol)), self.ctx.h,
                    "nnk_batch_set_refinement")

    _destroy = L.lib.nnk_batch_destroy  # held by the class: module globals may be gone at exit

    def __del__(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    @property
    def systems(self):
        return len(self.sizes) * self.nrhs

    def system(self, body, r):
        s = body * self.nrhs + r
        return slice(int(self.offsets[s]), int(self.offsets[s + 1]))

    def apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        L.check(L.lib.nnk_batch_apply(self.h, L.ptr(x), L.ptr(y), 0), self.ctx.h, "nnk_batch_apply")
        return y

    def solve(self, rhs, tol=1e-6, maxIter=200, restart=0):
        """x, per-system (flag, relres, iters) for the batch right-hand side."""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.empty_like(rhs)
        info = (L.SolveInfo * self.systems)()
        sp = L.SolveParams(float(tol), int(maxIter), int(restart))
        rc = L.lib.nnk_batch_solve(self.h, L.ptr(rhs), L.ptr(x), C.byref(sp), C.cast(info, C.c_void_p), 0)
        if rc not in (L.NNK_OK, L.NNK_E_NOCONV):
            L.check(rc, self.ctx.h, "nnk_batch_solve")
        return x, [(i.flag, i.relres, i.iters) for i in info]

    def modes_rhs(self, modes=RIGID_MODES):
        assert len(modes) == self.nrhs
        rhs = np.zeros(self.n)
        for b, N in enumerate(self.sizes):
            for r, m in enumerate(modes):
                rhs[self.system(b, r)] = mode_rhs(N, m)
        return rhs

    def solve_modes(self, tol=1e-6, maxIter=200, modes=RIGID_MODES):
        """Per body the 6 x 6 mobility matrix (column j = [U; Omega] for mode j)."""
        x, info = self.solve(self.modes_rhs(modes), tol=tol, maxIter=maxIter)
        out = []
        for b in range(len(self.sizes)):
            M = np.zeros((6, self.nrhs))
            for r in range(self.nrhs):
                M[:, r] = x[self.system(b, r)][-6:]
            out.append(M)
        return out, [info[b * self.nrhs:(b + 1) * self.nrhs] for b in range(len(self.sizes))]

    def profile(self, enable=True):
        L.check(L.lib.nnk_batch_profile(self.h, int(bool(enable))), self.ctx.h, "nnk_batch_profile")

    def profile_read(self, which=0):
        """{phase: ms} and {phase: launches} since the last read (which = 0:
        the batch's FMM, 1: the FP64 refinement FMM)."""
        ms = np.zeros(len(L.PHASES))
        ln = np.zeros(len(L.PHASES), np.int64)
        L.check(L.lib.nnk_batch_profile_read(self.h, int(which), L.ptr(ms), L.ptr(ln)), self.ctx.h,
                "nnk_batch_profile_read")
        return dict(zip(L.PHASES, ms)), dict(zip(L.PHASES, ln))

    def use_graphs(self, enable=True):
        """Replay the matvec from a CUDA graph (default) or launch kernel by kernel."""
        L.check(L.lib.nnk_batch_use_graphs(self.h, int(bool(enable))), self.ctx.h, "use_graphs")

    def set_deflation(self, enable=True):
        """Drop bodies whose right-hand sides all converged out of the forest
        FMM (default on; the solution is bitwise the same either way)."""
        L.check(L.lib.nnk_batch_set_deflation(self.h, int(bool(enable))), self.ctx.h, "set_deflation")

    def matvecs(self):
        c = C.c_int64()
        L.check(L.lib.nnk_batch_matvecs(self.h, C.byref(c)))
        return c.value
