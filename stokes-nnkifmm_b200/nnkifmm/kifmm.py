"""KIFMM: host mirror of Classes/KIFMM.m over the CUDA library.

    fmm = KIFMM(tree, [eps, mu], GMRES=1, format=2)
    vel = fmm.computeVel(potentials)

Same name-value options as KIFMM.m:50-60 (``GPU`` and ``parThreads`` are
accepted for compatibility; the work always runs on the GPU) plus
``precision``: 'fp64' (every step in FP64, the reference's operator),
'near32' (the same operator with the U-list P2P and X-list P2L, whose
sources are the forces themselves, in FP32) or 'mixed' (FP32 pairs, TF32
tensor-core M2L, Tikhonov-regularized check-to-equivalent operators).  Inputs may be numpy arrays (host) or
CUDA torch tensors (device); results come back the same way.
"""
import ctypes as C

import numpy as np

from . import _lib as L


class KIFMM:
    def __init__(self, tree, kernelPar, GPU=1, parThreads=0, blockSize=0.1, GMRES=0, coronaRes=6,
                 coronaShells=1, format=1, precision="fp64", reg=0.0, m2l="auto"):
        self.tree = tree
        self.ctx = tree.ctx
        eps, mu = float(kernelPar[0]), float(kernelPar[1])
        self.arguments = dict(GPU=GPU, parThreads=parThreads, blockSize=blockSize, GMRES=GMRES,
                              coronaRes=coronaRes, coronaShells=coronaShells, format=format,
                              kernelPar=(eps, mu), precision=precision)
        prec = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED, "near32": L.PREC_NEAR32}[precision]
        mode = {"auto": 0, "images": 1, "generate": 2, "pairs": 3, "fft": 4}[m2l]
        p = L.FmmParams(eps, mu, int(coronaRes), int(coronaShells), prec, mode, float(reg))
        h = C.c_void_p()
        L.check(L.lib.nnk_fmm_create(self.ctx.h, tree.h, C.byref(p), C.byref(h)), self.ctx.h, "KIFMM")
        self.h = h

    _destroy = L.lib.nnk_fmm_destroy  # held by the class: module globals may be gone at exit

    def __del__(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    # KIFMM.m:83-103: GMRES=1 -> vector; format 1 interleaved, 2 blocked
    def _layout(self):
        if self.arguments["GMRES"] == 1 and self.arguments["format"] == 2:
            return L.LAYOUT_BLOCKED
        return L.LAYOUT_ROWS

    def _call(self, fn, x, n_in, n_out, nrhs=1, extra=True):
        layout = self._layout()
        gm = self.arguments["GMRES"] == 1
        try:
            import torch
            is_t = isinstance(x, torch.Tensor)
        except ImportError:
            is_t = False
        if is_t:
            xin = x.contiguous().to(torch.float64)
            if not xin.is_cuda:
                raise ValueError("torch inputs must be CUDA tensors; pass numpy arrays for host data")
            if xin.device.index != self.ctx.device:
                raise ValueError(f"input on {xin.device}, the FMM on cuda:{self.ctx.device}")
            out = torch.empty(nrhs * 3 * n_out, dtype=torch.float64, device=xin.device)
            dev = 1
        else:
            xin = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
            out = np.empty(nrhs * 3 * n_out, dtype=np.float64)
            dev = 0
        nin = xin.numel() if is_t else xin.size
        if nin != nrhs * 3 * n_in:
            raise ValueError(f"expected {nrhs * 3 * n_in} values, got {nin}")
        args = [self.h, L.ptr(xin), L.ptr(out), layout]
        if extra:
            args.append(nrhs)
        args.append(dev)
        if is_t:
            # the library works on its context stream: order it after torch's
            # producers of xin, and torch's consumers of out after it
            torch.cuda.current_stream(xin.device).synchronize()
        L.check(fn(*args), self.ctx.h)
        if is_t:
            self.ctx.synchronize()
        if gm:
            return out if nrhs == 1 else out.reshape(nrhs, -1)
        return out.reshape(n_out, 3) if nrhs == 1 else out.reshape(nrhs, n_out, 3)

    def computeVel(self, potentials, nrhs=1):
        """KIFMM.computeVel (KIFMM.m:63-105)."""
        i = self.tree.info
        return self._call(L.lib.nnk_fmm_apply, potentials, i.num_potentials, i.num_targets, nrhs)

    def computeVelAdjoint(self, velocities, nrhs=1):
        """The exact transpose of computeVel: velocity-space input at the
        targets, potential-space output (<y, A x> = <A^T y, x>)."""
        i = self.tree.info
        return self._call(L.lib.nnk_fmm_apply_adjoint, velocities, i.num_targets, i.num_potentials, nrhs)

    def autotune(self, nrhs=1):
        """Pick the pair-kernel tile per launch group by timing; returns the
        summed pair-kernel milliseconds before and after."""
        a, b = C.c_double(), C.c_double()
        L.check(L.lib.nnk_fmm_autotune(self.h, int(nrhs), C.byref(a), C.byref(b)), self.ctx.h, "autotune")
        return a.value, b.value

    def setEps(self, eps):
        """Rebuild the eps-dependent operators for a new kernelPar(1)."""
        L.check(L.lib.nnk_fmm_set_eps(self.h, float(eps)), self.ctx.h, "setEps")
        self.arguments["kernelPar"] = (float(eps), self.arguments["kernelPar"][1])

    def setFold(self, mode=1):
        """Run the matvec's M2M and L2L folded into the check-to-equivalent
        products -- mode 1 where it pays (the default), 2 wherever available
        -- or, mode 0, as pair sums followed by those products;
        stats()["folded"] says whether the matvec folds."""
        L.check(L.lib.nnk_fmm_set_fold(self.h, int(mode)), self.ctx.h, "setFold")

    def setM2MForm(self, form=2):
        """M2M and L2L as products with their kernel matrices (2, the default
        where the tree allows it), M2M alone (1), or both as pair sums (0);
        stats()["m2m_product_pairs"] and ["l2l_product_pairs"] count what the
        products take over."""
        L.check(L.lib.nnk_fmm_set_m2m_form(self.h, int(form)), self.ctx.h, "setM2MForm")

    def setC2E(self, mode=1):
        """Check-to-equivalent products as one cuBLAS DGEMM per run of nodes
        sharing an operator (2, the default; forests and graph-captured
        matvecs use 0), as our FP64 SIMT products (0), on the tensor cores
        (1: int8 digit products with FP64 accuracy), or (-1) the fastest as
        timed by autotune()."""
        L.check(L.lib.nnk_fmm_set_c2e(self.h, int(mode)), self.ctx.h, "setC2E")

    def c2eMode(self):
        m = C.c_int32()
        L.check(L.lib.nnk_fmm_c2e_mode(self.h, C.byref(m)))
        return m.value

    def setup_times(self):
        """Host wall time (ms) of the set-up steps: points, tasks, m2l,
        operators, fold, total (nnk_fmm_setup_times)."""
        v = (C.c_double * 6)()
        L.check(L.lib.nnk_fmm_setup_times(self.h, v, 6))
        return dict(zip(("points", "tasks", "m2l", "operators", "fold", "total"), list(v)))

    def sourceCount(self):
        c = C.c_int64()
        L.check(L.lib.nnk_fmm_source_count(self.h, C.byref(c)))
        return c.value

    def gradPositions(self, forces, weights):
        """Gradient of <weights, computeVel(forces)> with respect to the target
        positions (n_tgt x 3) and the source positions (fine points in NEAREST
        mode, else the potentials; n x 3).  Host arrays in the KIFMM format."""
        i = self.tree.info
        f = np.ascontiguousarray(np.asarray(forces, np.float64).ravel())
        w = np.ascontiguousarray(np.asarray(weights, np.float64).ravel())
        if f.size != 3 * i.num_potentials or w.size != 3 * i.num_targets:
            raise ValueError("forces must hold 3 n_pot values and weights 3 n_tgt")
        gt = np.empty((i.num_targets, 3))
        gs = np.empty((self.sourceCount(), 3))
        L.check(L.lib.nnk_fmm_grad_positions(self.h, L.ptr(f), L.ptr(w), self._layout(), L.ptr(gt), L.ptr(gs), 0),
                self.ctx.h, "gradPositions")
        return gt, gs

    def computeVelSparse(self, potentials, nrhs=1):
        """KIFMM.computeVelSparse (KIFMM.m:107-155): coronaRes 4."""
        i = self.tree.info
        return self._call(L.lib.nnk_fmm_apply_sparse, potentials, i.num_potentials, i.num_targets, nrhs)

    def reducedComputeVel(self, potentials):
        """KIFMM.reducedComputeVel (KIFMM.m:157-198)."""
        i = self.tree.info
        return self._call(L.lib.nnk_fmm_reduced_apply, potentials, i.num_potentials, i.num_targets, extra=False)

    def reducedSolve(self, vel):
        """KIFMM.reducedSolve (KIFMM.m:200-242)."""
        i = self.tree.info
        return self._call(L.lib.nnk_fmm_reduced_solve, vel, i.num_targets, i.num_targets, extra=False)

    def stats(self):
        s = L.FmmStats()
        L.check(L.lib.nnk_fmm_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in L.FmmStats._fields_}

    def grad_eps(self, forces, weights):
        """weights^T (dF/deps) forces: the analytic eps-derivative of this FMM
        operator (FP64, exact check-to-equivalent inverses), nnk_fmm_grad_eps.
        forces (n_pot x 3) and weights (n_tgt x 3) as numpy arrays in the
        object's vector layout."""
        f = np.ascontiguousarray(np.asarray(forces, dtype=np.float64))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
        out = C.c_double()
        L.check(L.lib.nnk_fmm_grad_eps(self.h, L.ptr(f), L.ptr(w), self._layout(), C.byref(out), 0), self.ctx.h,
                "grad_eps")
        return out.value

    def profile(self, enable=True):
        """Per-phase CUDA-event timing of later computeVel calls."""
        L.check(L.lib.nnk_fmm_profile(self.h, int(bool(enable))))

    def profile_read(self):
        """{phase: (milliseconds, launches)} accumulated since the last read."""
        ms = np.zeros(len(L.PHASES))
        n = np.zeros(len(L.PHASES), np.int64)
        L.check(L.lib.nnk_fmm_profile_read(self.h, L.ptr(ms), L.ptr(n)), self.ctx.h)
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(L.PHASES)}

    def apply_raw(self, d_in, d_out, layout=L.LAYOUT_ROWS, on_device=1, nrhs=1):
        """computeVel on raw pointers (device or pinned host) without any
        Python-side staging; used by the benchmark."""
        L.check(L.lib.nnk_fmm_apply(self.h, d_in, d_out, layout, nrhs, on_device), self.ctx.h, "computeVel")

    def gmres(self, b, tol=1e-6, maxit=None, restart=0):
        """gmres(@(x) fmm.computeVel(x), b, [], tol, maxit) on the device
        (Data Generation/DirectMethodComparison.m:28).  Returns
        (x, flag, relres, iters) like MATLAB's first four outputs."""
        n = 3 * self.tree.info.num_targets
        bb = np.ascontiguousarray(np.asarray(b, dtype=np.float64).ravel())
        if bb.size != n:
            raise ValueError("rhs size")
        x = np.empty(n)
        sp_ = L.SolveParams(float(tol), int(maxit if maxit else min(n, 10)), int(restart))
        info = L.SolveInfo()
        rc = L.lib.nnk_fmm_solve(self.h, L.ptr(bb), L.ptr(x), self._layout(), C.byref(sp_), C.byref(info), 0)
        if rc not in (L.NNK_OK, L.NNK_E_NOCONV):
            L.check(rc, self.ctx.h, "gmres")
        return x, info.flag, info.relres, info.iters
