"""OcTree: host mirror of Classes/OcTree.m over nnk_tree_build.

Same constructor arguments and property names as the reference (OcTree.m:59-95);
node ids, pointIndex and the interaction lists are the reference's 1-based
ids.  The build errors with MaxDepthError('Max level reached: Increase Max
Depth') exactly when the reference does (OcTree.m:168-170).
"""
import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _lib as L


def _as_points(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, 3))
    return a


class OcTree:
    def __init__(self, potPoints, targetPoints, parThreads=0, nodeCapacity=200, maxDepth=21,
                 finePoints=None, nearest=0, NN=None, blockSize=0.2, device=0, ctx=None, builder="auto"):
        self.ctx = ctx if ctx is not None else L.context(device)
        pot = _as_points(potPoints)
        same = targetPoints is potPoints or (np.shape(targetPoints) == np.shape(potPoints)
                                             and np.array_equal(np.asarray(targetPoints), np.asarray(potPoints)))
        tgt = pot if same else _as_points(targetPoints)
        self.arguments = dict(parThreads=parThreads, nodeCapacity=nodeCapacity, maxDepth=maxDepth,
                              nearest=int(bool(nearest)), blockSize=blockSize)
        fine = None
        rp = col = val = None
        q = 0
        if nearest:
            if finePoints is None:
                raise ValueError("nearest=1 needs finePoints")
            fine = _as_points(finePoints)
            q = fine.shape[0]
            if NN is not None:
                nn = sp.csr_matrix(NN)
                nn.sort_indices()
                rp = np.ascontiguousarray(nn.indptr.astype(np.int64))
                col = np.ascontiguousarray(nn.indices.astype(np.int32))
                val = np.ascontiguousarray(nn.data.astype(np.float64))
        # where the node structure and NN are built: auto (GPU when present), host, gpu
        params = L.TreeParams(int(nodeCapacity), int(maxDepth), int(bool(nearest)),
                              {"auto": 0, "host": 1, "gpu": 2}[builder])
        h = C.c_void_p()
        rc = L.lib.nnk_tree_build(self.ctx.h, L.ptr(pot), pot.shape[0], L.ptr(tgt), tgt.shape[0],
                                  L.ptr(fine), q, L.ptr(rp), L.ptr(col), L.ptr(val),
                                  C.byref(params), C.byref(h))
        L.check(rc, self.ctx.h, "OcTree")
        self.h = h
        info = L.TreeInfo()
        L.check(L.lib.nnk_tree_info_get(self.h, C.byref(info)))
        self.info = info
        self.nodeCount = info.node_count
        self.nodeCapacity = info.node_capacity
        self.finePoints = fine if nearest else None
        self._nn = sp.csr_matrix(NN) if (nearest and NN is not None) else None
        self._cache = {}

    _destroy = L.lib.nnk_tree_destroy  # held by the class: module globals may be gone at exit

    def __del__(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    # ---- exported arrays (lazy)
    def _nodes(self):
        if "nodes" not in self._cache:
            n = self.nodeCount
            lvl = np.zeros(n, np.int32)
            par = np.zeros(n, np.int32)
            ch = np.zeros((n, 8), np.int32)
            cor = np.zeros((n, 6), np.float64)
            pi = np.zeros(self.info.num_points, np.int32)
            L.check(L.lib.nnk_tree_export_nodes(self.h, L.ptr(lvl), L.ptr(par), L.ptr(ch), L.ptr(cor), L.ptr(pi)))
            self._cache["nodes"] = (lvl, par, ch, cor, pi)
        return self._cache["nodes"]

    @property
    def nodeLevel(self):
        return self._nodes()[0]

    @property
    def nodeParents(self):
        return self._nodes()[1]

    @property
    def nodeChildren(self):
        return self._nodes()[2]

    @property
    def nodeCorners(self):
        return self._nodes()[3]

    @property
    def pointIndex(self):
        return self._nodes()[4]

    def _points(self):
        if "points" not in self._cache:
            n = self.info.num_points
            pts = np.zeros((n, 3))
            pm = np.zeros(n, np.uint8)
            tm = np.zeros(n, np.uint8)
            L.check(L.lib.nnk_tree_export_points(self.h, L.ptr(pts), L.ptr(pm), L.ptr(tm)))
            self._cache["points"] = (pts, pm.astype(bool), tm.astype(bool))
        return self._cache["points"]

    @property
    def points(self):
        return self._points()[0]

    @property
    def NN(self):
        """tree.NN (Q x N, NEAREST mode): the matrix given, or the one the tree
        was built with (recomputed here bit for bit; both builders are exact)."""
        if self.finePoints is None:
            return None
        if self._nn is None:
            self._nn = nearestMatrix(self.points, self.finePoints, device=self.ctx.device)
        return self._nn

    @property
    def potentials(self):
        return self._points()[1]

    @property
    def targets(self):
        return self._points()[2]

    def interaction_list(self, which):
        """CSR (offsets, ids) of tree.interactions(:,which+1); which 0 U, 1 V, 2 W, 3 X."""
        key = ("list", which)
        if key not in self._cache:
            tot = [self.info.u_total, self.info.v_total, self.info.w_total, self.info.x_total][which]
            off = np.zeros(self.nodeCount + 1, np.int64)
            ids = np.zeros(max(tot, 1), np.int32)
            L.check(L.lib.nnk_tree_export_list(self.h, which, L.ptr(off), L.ptr(ids)))
            self._cache[key] = (off, ids[:tot])
        return self._cache[key]

    @property
    def interactions(self):
        """tree.interactions as a list of [U, V, W, X] per node (index = id - 1)."""
        lists = [self.interaction_list(k) for k in range(4)]
        out = []
        for i in range(self.nodeCount):
            out.append([ids[off[i]:off[i + 1]] for off, ids in lists])
        return out

    def getPotentialPoints(self):
        return self.points[self.potentials]

    def getTargetPoints(self):
        return self.points[self.targets]

    def getFinePoints(self):
        return self.finePoints


def nearestMatrix(coarse, fine, blockSize=0.2, threads=0, device=0, builder="auto", ties="share"):
    """nearestMatrix (Tools/Nearest/nearestMatrix.m:17-41) through the library:
    returns the (Q x N) scipy CSR matrix with exact FP64 ties sharing 1/k
    (on the GPU when there is one, or on the host with builder="host").

    ties="reference" gives the tie weights as nearestMatrix.m writes them
    (per block of floor(blockSize 2^27 / (9 Q)) fine points, the tied pairs in
    column-major order take the 1/k weights in row-major order, so rows with
    ties need not sum to one); the default "share" keeps 1/k per tied pair."""
    if ties not in ("share", "reference"):
        raise ValueError("ties must be 'share' or 'reference'")
    ctx = L.context(device)
    fn = L.lib.nnk_nearest_matrix_host if builder == "host" else L.lib.nnk_nearest_matrix
    c = _as_points(coarse)
    f = _as_points(fine)
    nnz = C.c_int64()
    L.check(fn(ctx.h, L.ptr(c), c.shape[0], L.ptr(f), f.shape[0], C.byref(nnz), None, None, None), ctx.h,
            "nearestMatrix")
    rp = np.zeros(f.shape[0] + 1, np.int64)
    col = np.zeros(max(nnz.value, 1), np.int32)
    val = np.zeros(max(nnz.value, 1), np.float64)
    L.check(fn(ctx.h, L.ptr(c), c.shape[0], L.ptr(f), f.shape[0], C.byref(nnz), L.ptr(rp), L.ptr(col), L.ptr(val)),
            ctx.h, "nearestMatrix")
    if ties == "reference":
        L.check(L.lib.nnk_nearest_reference_weights(ctx.h, f.shape[0], L.ptr(rp), L.ptr(col), L.ptr(val),
                                                     float(blockSize)), ctx.h, "nearestMatrix")
    return sp.csr_matrix((val[:nnz.value], col[:nnz.value], rp), shape=(f.shape[0], c.shape[0]))
